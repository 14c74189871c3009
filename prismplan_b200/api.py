"""Python API over the C ABI (torch tensors in, torch tensors out).

Reference-facing calls keep the reference's names and semantics:
  * ``check_collision_scene(configs, scene, robot, collision_margin)``
    -- prrtc.check_collision_scene (code/gpu_planning/cpp/src/python/
    bindings.cpp:493-532): host numpy in, host bool numpy out, synchronous.
  * ``EdgeEvalGpu(dim, max_edges, scene, model).evaluate(...)``
    -- ppln::search::EdgeEvalGpu (cpp/src/planning/edge_batch_bridge.hh:27-111).
Device-resident torch calls (``check_configs``, ``check_edges``,
``traj_cost``, ``rollout_costs``) are asynchronous on the current stream.
``hinge_cost`` applies a torch.autograd.Function whose backward is the
fused hand-written adjoint.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from . import _lib
from .robot import RobotModelBuilder
from .scene import SceneCollisionDataBuilder, SceneTensors


def _torch():
    import torch

    return torch


def _view(scene) -> _lib.SceneView:
    if scene is None:
        return SceneCollisionDataBuilder().build()
    if isinstance(scene, SceneTensors):
        return scene.view()
    if isinstance(scene, SceneCollisionDataBuilder):
        return scene.build()
    if isinstance(scene, _lib.SceneView):
        return scene
    raise TypeError(f"unsupported scene type {type(scene).__name__}")


def _dev_f32(t, shape_last=None):
    torch = _torch()
    if not isinstance(t, torch.Tensor):
        t = torch.as_tensor(np.asarray(t, np.float32))
    if not t.is_cuda:
        t = t.cuda()
    t = t.to(torch.float32).contiguous()
    if shape_last is not None and t.shape[-1] != shape_last:
        raise ValueError(f"last dimension must be {shape_last}, got {tuple(t.shape)}")
    return t


def _stream(stream):
    return _lib.stream_handle(stream)


def _model(robot: RobotModelBuilder) -> C.c_void_p:
    return robot.handle


# ---------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------
def _config_flags(clearance, check_self, no_gate, blocks_per_sm=0):
    flags = 0
    if clearance in ("obb", "both"):
        flags |= _lib.PS_CLEARANCE_OBB
    if clearance in ("esdf", "both"):
        flags |= _lib.PS_CLEARANCE_ESDF
    if check_self:
        flags |= _lib.PS_CHECK_SELF
    if no_gate:
        flags |= _lib.PS_NO_GATE
    return flags | _lib.PS_CONFIG_BLOCKS_PER_SM(blocks_per_sm)


def check_configs(robot: RobotModelBuilder, scene, q, collision_margin: float = 0.0,
                  clearance: Optional[str] = None, check_self: bool = False,
                  no_gate: bool = False, stream=None, blocks_per_sm: int = 0):
    """Two-phase any-collision for every row of ``q`` [N, n_dof] (CUDA).

    ``clearance``: None, "obb", "esdf" or "both" -- min over spheres of the
    selected signed clearance (radius + margin), 1000.0 when nothing applies.
    ``blocks_per_sm``: grid of the kernel (0 = default; tune_configs picks
    it). Returns (hit uint8 [N], clearance float32 [N] or None)."""
    torch = _torch()
    q = _dev_f32(q, robot.n_dof)
    n = q.shape[0]
    hit = torch.empty(n, dtype=torch.uint8, device=q.device)
    flags = _config_flags(clearance, check_self, no_gate, blocks_per_sm)
    clr = torch.empty(n, dtype=torch.float32, device=q.device) if clearance else None
    v = _view(scene)
    _lib.check(_lib.load().ps_check_configs(
        _model(robot), C.byref(v), q.data_ptr(), n, float(collision_margin), flags,
        hit.data_ptr(), clr.data_ptr() if clr is not None else None, _stream(stream)))
    return hit, clr


def check_collision_scene(configs, scene, robot: RobotModelBuilder,
                          collision_margin: float = 0.0) -> np.ndarray:
    """Drop-in for prrtc.check_collision_scene (bindings.cpp:493-532), same
    keywords: configs [N, n_dof] host array -> bool [N] (True = in
    collision), synchronous. Raises RuntimeError on a column mismatch, as the
    reference does (bindings.cpp:505-507)."""
    scene_builder = scene
    torch = _torch()
    robot.build()
    c = np.asarray(configs, np.float32)
    if c.ndim != 2 or c.shape[1] != robot.n_dof:
        raise RuntimeError("configs columns mismatch with robot n_dof")
    if c.shape[0] == 0:
        return np.zeros(0, bool)
    hit, _ = check_configs(robot, scene_builder, torch.from_numpy(c).cuda(), collision_margin)
    return hit.cpu().numpy().astype(bool)


def fk_spheres(robot: RobotModelBuilder, q, stream=None):
    """World sphere centres [N, n_spheres, 3] (descriptor order)."""
    torch = _torch()
    q = _dev_f32(q, robot.n_dof)
    n = q.shape[0]
    out = torch.empty((n, len(robot.sphere_to_joint), 3), dtype=torch.float32, device=q.device)
    _lib.check(_lib.load().ps_fk_spheres(_model(robot), q.data_ptr(), n, out.data_ptr(), _stream(stream)))
    return out


# ---------------------------------------------------------------------------
# edges
# ---------------------------------------------------------------------------
@dataclass
class EdgeEvalParams:
    """ppln::search::EdgeEvalParams (edge_eval.cuh:37-51) plus the L-inf rule."""

    granularity: int = 16
    collision_margin: float = 0.0
    check_self: bool = False
    compute_clearance: bool = False
    enable_mesh: bool = False
    resolution: float = 0.0
    max_joint_step: float = 0.0
    max_samples: int = 1024
    time_budget_ms: float = 0.0   # persistent paths: stop after this much device time (0 = none)
    # launch shape of the persistent paths (0 = automatic; tune_edges picks them)
    probe: int = 0                # 0 automatic, 1 on, 2 off
    queue_blocks_per_sm: int = 0  # 0 = all that fit
    grab: int = 0                 # queue items per grab, 0 = automatic

    def to_c(self) -> _lib.EdgeParams:
        if self.enable_mesh:
            raise ValueError("mesh edge checks are not supported (enable_mesh must be False)")
        p = _lib.EdgeParams()
        p.granularity = int(self.granularity)
        p.resolution = float(self.resolution)
        p.max_joint_step = float(self.max_joint_step)
        p.max_samples = int(self.max_samples)
        p.collision_margin = float(self.collision_margin)
        p.check_self = int(bool(self.check_self))
        p.compute_clearance = int(bool(self.compute_clearance))
        p.time_budget_ms = float(self.time_budget_ms)
        p.probe = int(self.probe)
        p.queue_blocks_per_sm = int(self.queue_blocks_per_sm)
        p.grab = int(self.grab)
        return p


def edges_workspace(n_edges: int, device="cuda"):
    torch = _torch()
    nbytes = int(_lib.load().ps_edges_workspace_bytes(int(n_edges)))
    return torch.empty(nbytes, dtype=torch.uint8, device=device)


def edges_status(workspace=None) -> int:
    """PS_OK or PS_ETIMEOUT for the last persistent call on ``workspace``
    (None: the built-in workspace of the current device). Synchronous."""
    st = C.c_int(0)
    _lib.check(_lib.load().ps_edges_status(workspace.data_ptr() if workspace is not None else None, C.byref(st)))
    return st.value


def check_edges(robot: RobotModelBuilder, scene, frm, to, samples=None,
                params: Optional[EdgeEvalParams] = None, persistent: bool = True,
                workspace=None, out=None, stream=None):
    """Edge validity for rows of ``frm``/``to`` [E, n_dof] (CUDA).

    ``samples`` [E] int32 (optional) fixes G per edge; otherwise ``params``
    decides (resolution / max_joint_step / granularity). Returns
    (valid uint8 [E], cost float32 [E], clearance float32 [E])."""
    torch = _torch()
    params = params or EdgeEvalParams()
    frm = _dev_f32(frm, robot.n_dof)
    to = _dev_f32(to, robot.n_dof)
    E = frm.shape[0]
    if to.shape[0] != E:
        raise ValueError("from/to row counts differ")
    if samples is not None:
        samples = torch.as_tensor(samples).to(device=frm.device, dtype=torch.int32).contiguous()
        if samples.shape[0] != E:
            raise ValueError("samples must have one entry per edge")
    if out is None:
        valid = torch.empty(E, dtype=torch.uint8, device=frm.device)
        cost = torch.empty(E, dtype=torch.float32, device=frm.device)
        clr = torch.empty(E, dtype=torch.float32, device=frm.device)
    else:
        valid, cost, clr = out
    p = params.to_c()
    v = _view(scene)
    lib = _lib.load()
    sp = samples.data_ptr() if samples is not None else None
    if persistent:
        if workspace is None:
            workspace = edges_workspace(E, frm.device)
        _lib.check(lib.ps_check_edges(_model(robot), C.byref(v), frm.data_ptr(), to.data_ptr(), sp, E,
                                      C.byref(p), valid.data_ptr(), cost.data_ptr(), clr.data_ptr(),
                                      workspace.data_ptr(), workspace.numel(), _stream(stream)))
    else:
        _lib.check(lib.ps_check_edges_plain(_model(robot), C.byref(v), frm.data_ptr(), to.data_ptr(), sp, E,
                                            C.byref(p), valid.data_ptr(), cost.data_ptr(), clr.data_ptr(),
                                            _stream(stream)))
    return valid, cost, clr


def tune_edges(robot: RobotModelBuilder, scene, frm, to, samples=None, params: Optional[EdgeEvalParams] = None,
               stream=None):
    """Autotune the persistent edge path's launch shape (ps_tune_edges) on
    these edges. Returns (params with probe / queue_blocks_per_sm / grab set,
    {"probe", "queue_blocks_per_sm", "grab", "best_ms", "default_ms",
    "candidates"})."""
    import copy

    torch = _torch()
    params = params or EdgeEvalParams()
    frm = _dev_f32(frm, robot.n_dof)
    to = _dev_f32(to, robot.n_dof)
    E = frm.shape[0]
    if samples is not None:
        samples = torch.as_tensor(samples).to(device=frm.device, dtype=torch.int32).contiguous()
    valid = torch.empty(E, dtype=torch.uint8, device=frm.device)
    cost = torch.empty(E, dtype=torch.float32, device=frm.device)
    clr = torch.empty(E, dtype=torch.float32, device=frm.device)
    ws = edges_workspace(E, frm.device)
    p = params.to_c()
    tuned = _lib.EdgeParams()
    info = _lib.EdgeTuning()
    v = _view(scene)
    _lib.check(_lib.load().ps_tune_edges(_model(robot), C.byref(v), frm.data_ptr(), to.data_ptr(),
                                         samples.data_ptr() if samples is not None else None, E, C.byref(p),
                                         valid.data_ptr(), cost.data_ptr(), clr.data_ptr(), ws.data_ptr(),
                                         ws.numel(), _stream(stream), C.byref(info), C.byref(tuned)))
    out = copy.copy(params)
    out.probe, out.queue_blocks_per_sm, out.grab = tuned.probe, tuned.queue_blocks_per_sm, tuned.grab
    return out, {name: getattr(info, name) for name, _ in info._fields_}


def tune_configs(robot: RobotModelBuilder, scene, q, collision_margin: float = 0.0, clearance: Optional[str] = None,
                 check_self: bool = False, stream=None):
    """Autotune the configuration kernel's grid (ps_tune_configs). Returns
    (blocks_per_sm to pass to check_configs, {"blocks_per_sm", "best_ms",
    "default_ms", "candidates"})."""
    torch = _torch()
    q = _dev_f32(q, robot.n_dof)
    n = q.shape[0]
    flags = _config_flags(clearance, check_self, False)
    hit = torch.empty(n, dtype=torch.uint8, device=q.device)
    clr = torch.empty(n, dtype=torch.float32, device=q.device) if clearance else None
    info = _lib.ConfigTuning()
    tuned = C.c_uint(0)
    v = _view(scene)
    _lib.check(_lib.load().ps_tune_configs(_model(robot), C.byref(v), q.data_ptr(), n, float(collision_margin), flags,
                                           hit.data_ptr(), clr.data_ptr() if clr is not None else None,
                                           _stream(stream), C.byref(info), C.byref(tuned)))
    return info.blocks_per_sm, {name: getattr(info, name) for name, _ in info._fields_}


class EdgeEvalGpu:
    """Drop-in for ppln::search::EdgeEvalGpu (edge_batch_bridge.hh:27-111)
    over the library's native bridge (ps_edge_bridge_*): device buffers,
    pinned host mirrors, the persistent path's workspace and a private stream
    owned by the library. ``evaluate`` hands the host arrays to the bridge,
    which stages them into its pinned mirrors (OpenMP threads), copies them
    in, runs the persistent edge check from a CUDA graph per (num_edges,
    params), copies the outputs back and synchronises. The scene is held as built at
    construction, like the reference's by-value SceneCollisionData;
    ``set_scene`` replaces it. Raises on num_edges > max_edges like the
    reference (:67-68)."""

    def __init__(self, dim: int, max_edges: int, scene, model: RobotModelBuilder):
        self.dim, self.max_edges, self.scene, self.model = int(dim), int(max_edges), scene, model
        if model.n_dof != self.dim:
            raise ValueError("dim must equal the robot's n_dof")
        self._lib = _lib.load()
        self._view = _view(scene)
        h = C.c_void_p()
        _lib.check(self._lib.ps_edge_bridge_create(_model(model), C.byref(self._view), self.dim, self.max_edges,
                                                   C.byref(h)))
        self._h = h
        self._params_key = None
        self._params_c = None
        self._pending = {}

    def host_inputs(self):
        """The bridge's pinned input mirrors (slot 0) as numpy arrays
        (from, to: [max_edges, dim] float32), valid until ``close``. Edges
        written there and passed to ``evaluate`` as ``from_flat`` / ``to_flat``
        go to the device without a staging copy."""
        if getattr(self, "_views", None) is None:
            pf, pt = C.c_void_p(), C.c_void_p()
            _lib.check(self._lib.ps_edge_bridge_host_inputs(self._h, C.byref(pf), C.byref(pt)))
            shape = (self.max_edges, self.dim)
            self._views = (np.ctypeslib.as_array(C.cast(pf, C.POINTER(C.c_float)), shape=shape),
                           np.ctypeslib.as_array(C.cast(pt, C.POINTER(C.c_float)), shape=shape))
        return self._views

    def set_scene(self, scene) -> None:
        """Use another scene (its tensors must outlive the calls)."""
        view = _view(scene)
        _lib.check(self._lib.ps_edge_bridge_set_scene(self._h, C.byref(view)))
        self.scene, self._view = scene, view

    def evaluate(self, from_flat, to_flat, num_edges: int, params: EdgeEvalParams):
        """Copy in, check, copy out, synchronise; returns host arrays
        (valid uint8 [n], cost float32 [n], clearance float32 [n] when
        params.compute_clearance else empty)."""
        n = int(num_edges)
        if n <= 0:
            return np.zeros(0, np.uint8), np.zeros(0, np.float32), np.zeros(0, np.float32)
        if n > self.max_edges:
            raise RuntimeError("EdgeEvalGpu: num_edges exceeds max_edges_")
        f = np.ascontiguousarray(from_flat, dtype=np.float32)
        t = np.ascontiguousarray(to_flat, dtype=np.float32)
        k = n * self.dim
        if f.size < k or t.size < k:
            raise ValueError("from_flat/to_flat hold fewer than num_edges * dim values")
        key = tuple(vars(params).values())
        if key != self._params_key:
            self._params_c, self._params_key = params.to_c(), key
        valid = np.empty(n, np.uint8)
        cost = np.empty(n, np.float32)
        clr = np.empty(n, np.float32) if params.compute_clearance else np.zeros(0, np.float32)
        _lib.check(self._lib.ps_edge_bridge_evaluate(self._h, f.ctypes.data, t.ctypes.data, n,
                                                     C.byref(self._params_c), valid.ctypes.data, cost.ctypes.data,
                                                     clr.ctypes.data if params.compute_clearance else None))
        return valid, cost, clr

    def submit(self, from_flat, to_flat, num_edges: int, params: EdgeEvalParams, slot: int = 0) -> int:
        """Asynchronous half of ``evaluate`` on one of the bridge's two slots:
        stages the host arrays (they may be reused on return) and queues the
        copy in, the check and the copy out. ``wait(slot)`` returns the
        outputs. While the GPU checks one slot's batch, the host can stage and
        submit the other's."""
        n = int(num_edges)
        if n > self.max_edges:
            raise RuntimeError("EdgeEvalGpu: num_edges exceeds max_edges_")
        if slot in self._pending:
            raise RuntimeError(f"EdgeEvalGpu: slot {slot} has a call not yet waited for")
        f = np.ascontiguousarray(from_flat, dtype=np.float32)
        t = np.ascontiguousarray(to_flat, dtype=np.float32)
        if n > 0 and (f.size < n * self.dim or t.size < n * self.dim):
            raise ValueError("from_flat/to_flat hold fewer than num_edges * dim values")
        key = tuple(vars(params).values())
        if key != self._params_key:
            self._params_c, self._params_key = params.to_c(), key
        _lib.check(self._lib.ps_edge_bridge_submit(self._h, int(slot), f.ctypes.data, t.ctypes.data, n,
                                                   C.byref(self._params_c)))
        self._pending[slot] = (max(n, 0), bool(params.compute_clearance))
        return slot

    def wait(self, slot: int = 0):
        """Outputs of the call submitted to ``slot`` (as ``evaluate`` returns them)."""
        if slot not in self._pending:
            raise RuntimeError(f"EdgeEvalGpu: slot {slot} has no call to wait for")
        n, want_clr = self._pending.pop(slot)
        valid = np.empty(n, np.uint8)
        cost = np.empty(n, np.float32)
        clr = np.empty(n, np.float32) if want_clr else np.zeros(0, np.float32)
        _lib.check(self._lib.ps_edge_bridge_wait(self._h, int(slot), valid.ctypes.data, cost.ctypes.data,
                                                 clr.ctypes.data if want_clr else None))
        return valid, cost, clr

    def status(self) -> int:
        """PS_ETIMEOUT when the time budget of the call waited for last ran out, else PS_OK."""
        code = C.c_int(0)
        _lib.check(self._lib.ps_edge_bridge_status(self._h, C.byref(code)))
        return code.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._views = None   # views of the mirrors the destroy frees
            self._lib.ps_edge_bridge_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# trajectory costs
# ---------------------------------------------------------------------------
@dataclass
class CostParams:
    """Hinge / smoothness parameters (CHOMP_settings.hh:35-46 names)."""

    collision_cost_weight: float = 20.0
    world_collision_margin: float = 0.02
    self_collision_margin: float = 0.01
    include_self: bool = True
    smoothness_weight: float = 0.0
    delta_t: float = 0.1

    def to_c(self, layout: int) -> _lib.CostParams:
        p = _lib.CostParams()
        p.collision_cost_weight = float(self.collision_cost_weight)
        p.world_margin = float(self.world_collision_margin)
        p.self_margin = float(self.self_collision_margin)
        p.include_self = int(bool(self.include_self))
        p.smoothness_weight = float(self.smoothness_weight)
        p.delta_t = float(self.delta_t)
        p.layout = int(layout)
        return p


def traj_cost(robot: RobotModelBuilder, scene, q, params: Optional[CostParams] = None,
              want_grad: bool = True, want_waypoint: bool = True, layout: int = _lib.PS_LAYOUT_BTD,
              stream=None):
    """Summed-hinge (+ self hinge, + smoothness) cost of trajectories ``q``
    [B, T, n_dof] (or [B, n_dof, T] with PS_LAYOUT_BDT), one fused launch for
    cost and gradient. Returns (waypoint_cost [B, T] or None, traj_cost [B],
    grad like q or None)."""
    torch = _torch()
    params = params or CostParams()
    q = _dev_f32(q)
    if q.dim() != 3:
        raise ValueError("q must be 3-D")
    if layout == _lib.PS_LAYOUT_BTD:
        B, T, D = q.shape
    else:
        B, D, T = q.shape
    if D != robot.n_dof:
        raise ValueError("DoF dimension mismatch")
    wp = torch.empty((B, T), dtype=torch.float32, device=q.device) if want_waypoint else None
    tc = torch.empty(B, dtype=torch.float32, device=q.device)
    g = torch.empty_like(q) if want_grad else None
    p = params.to_c(layout)
    v = _view(scene)
    _lib.check(_lib.load().ps_traj_cost(_model(robot), C.byref(v), q.data_ptr(), B, T, C.byref(p),
                                        wp.data_ptr() if wp is not None else None, tc.data_ptr(),
                                        g.data_ptr() if g is not None else None, _stream(stream)))
    return wp, tc, g


def rollout_costs(robot: RobotModelBuilder, scene, rollouts, params: Optional[CostParams] = None,
                  broadcast_d: bool = False, stream=None):
    """STOMP per-(rollout, waypoint) state cost of ``rollouts`` [R, n_dof, T]
    (the reference layout). Returns [R, T] or, with broadcast_d, [R, n_dof, T]
    as stomp_state_cost_kernel writes it."""
    torch = _torch()
    params = params or CostParams()
    r = _dev_f32(rollouts)
    R, D, T = r.shape
    if D != robot.n_dof:
        raise ValueError("DoF dimension mismatch")
    out = torch.empty((R, D, T) if broadcast_d else (R, T), dtype=torch.float32, device=r.device)
    p = params.to_c(_lib.PS_LAYOUT_BDT)
    v = _view(scene)
    _lib.check(_lib.load().ps_rollout_costs(_model(robot), C.byref(v), r.data_ptr(), R, T, C.byref(p),
                                            int(bool(broadcast_d)), out.data_ptr(), _stream(stream)))
    return out


# ---------------------------------------------------------------------------
# batched CHOMP optimisation
# ---------------------------------------------------------------------------
@dataclass
class ChompSettings:
    """CHOMP settings with the reference's names and defaults
    (cpp/src/planning/CHOMP_settings.hh:23-55; time_limit_ms and
    collision_margin from pRRTC_settings.hh:6,25). ``fd_epsilon`` has no
    counterpart: the obstacle gradient is the exact adjoint."""

    num_timesteps: int = 51
    num_iterations: int = 100
    num_iterations_after_valid: int = 5
    step_size: float = 0.3
    smoothness_weight: float = 1.0
    collision_cost_weight: float = 20.0
    world_collision_margin: float = 0.02
    self_collision_margin: float = 0.01
    delta_t: float = 0.1
    convergence_eps: float = 1.0e-4
    collision_check_step: float = 0.05
    collision_margin: float = 0.0
    time_limit_ms: float = 4000.0
    include_self: bool = True
    check_self: bool = True

    def to_c(self) -> _lib.ChompParams:
        p = _lib.ChompParams()
        p.num_iterations = int(self.num_iterations)
        p.num_iterations_after_valid = int(self.num_iterations_after_valid)
        p.step_size = float(self.step_size)
        p.smoothness_weight = float(self.smoothness_weight)
        p.collision_cost_weight = float(self.collision_cost_weight)
        p.world_margin = float(self.world_collision_margin)
        p.self_margin = float(self.self_collision_margin)
        p.delta_t = float(self.delta_t)
        p.convergence_eps = float(self.convergence_eps)
        p.collision_check_step = float(self.collision_check_step)
        p.collision_margin = float(self.collision_margin)
        p.include_self = int(bool(self.include_self))
        p.check_self = int(bool(self.check_self))
        p.time_limit_ms = float(self.time_limit_ms)
        return p


@dataclass
class ChompResult:
    """Per-request outcome of ``chomp_optimize`` / ``chomp_solve``, the fields
    of CHOMPResult (Planners.hh) for B requests at once."""

    path: "torch.Tensor"        # [B, T, D] best valid iterate (last iterate if none)
    solved: "torch.Tensor"      # [B] bool
    iterations: "torch.Tensor"  # [B] int32, updates applied
    cost: "torch.Tensor"        # [B] total cost of ``path``
    theta: "torch.Tensor"       # [B, T, D] last iterate


def chomp_workspace(robot: RobotModelBuilder, B: int, T: int, device="cuda"):
    torch = _torch()
    nbytes = int(_lib.load().ps_chomp_workspace_bytes(_model(robot), int(B), int(T)))
    return torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device)


def chomp_linear_init(robot: RobotModelBuilder, starts, goals, T: int):
    """Straight-line initial trajectories [B, T, D] clamped to the joint
    limits, as chomp_init_trajectory_kernel (chomp.cu:57-69) builds them."""
    torch = _torch()
    s = _dev_f32(starts, robot.n_dof).reshape(-1, robot.n_dof)
    g = _dev_f32(goals, robot.n_dof).reshape(-1, robot.n_dof)
    if s.shape != g.shape:
        raise ValueError("starts and goals differ in shape")
    t = torch.arange(T, device=s.device, dtype=torch.float32)
    frac = t / float(T - 1) if T > 1 else torch.zeros_like(t)
    v = s[:, None, :] * (1.0 - frac)[None, :, None] + g[:, None, :] * frac[None, :, None]
    lo = torch.tensor(np.asarray(robot.joint_lower, np.float32), device=s.device)
    hi = torch.tensor(np.asarray(robot.joint_upper, np.float32), device=s.device)
    return torch.maximum(lo, torch.minimum(hi, v)).contiguous()


def chomp_optimize(robot: RobotModelBuilder, scene, theta, settings: Optional[ChompSettings] = None,
                   workspace=None, stream=None) -> ChompResult:
    """Run CHOMP on B trajectories ``theta`` [B, T, D] at once (the reference
    runs one, chomp.cu:358-600). ``theta`` is updated in place when it is a
    contiguous float32 CUDA tensor. Synchronises the stream every 8
    iterations."""
    torch = _torch()
    settings = settings or ChompSettings()
    th = _dev_f32(theta)
    if th.dim() != 3 or th.shape[2] != robot.n_dof:
        raise ValueError("theta must be [B, T, n_dof]")
    B, T, D = th.shape
    best = torch.empty_like(th)
    solved = torch.empty(B, dtype=torch.uint8, device=th.device)
    iters = torch.empty(B, dtype=torch.int32, device=th.device)
    cost = torch.empty(B, dtype=torch.float32, device=th.device)
    ws = workspace if workspace is not None else chomp_workspace(robot, B, T, th.device)
    p = settings.to_c()
    v = _view(scene)
    _lib.check(_lib.load().ps_chomp_optimize(_model(robot), C.byref(v), th.data_ptr(), B, T, C.byref(p),
                                             best.data_ptr(), solved.data_ptr(), iters.data_ptr(),
                                             cost.data_ptr(), ws.data_ptr(), ws.numel(), _stream(stream)))
    return ChompResult(best, solved.bool(), iters, cost, th)


def chomp_solve(robot: RobotModelBuilder, scene, starts, goals, settings: Optional[ChompSettings] = None,
                stream=None) -> ChompResult:
    """CHOMP::solve_runtime_scene for B (start, goal) pairs: straight-line
    initialisation over num_timesteps waypoints, the optimiser loop, and the
    path's first and last waypoints set to start and goal
    (chomp.cu:557-567)."""
    settings = settings or ChompSettings()
    theta = chomp_linear_init(robot, starts, goals, settings.num_timesteps)
    res = chomp_optimize(robot, scene, theta, settings, stream=stream)
    res.path[:, 0, :] = _dev_f32(starts, robot.n_dof).reshape(-1, robot.n_dof)
    res.path[:, -1, :] = _dev_f32(goals, robot.n_dof).reshape(-1, robot.n_dof)
    return res


# ---------------------------------------------------------------------------
# batched STOMP optimisation
# ---------------------------------------------------------------------------
@dataclass
class StompSettings:
    """STOMP settings with the reference's names and defaults
    (cpp/src/planning/STOMP_settings.hh:17-59; time_limit_ms and
    collision_margin from pRRTC_settings.hh:6,25). ``seed`` keys the noise
    stream (the reference's fixed seed is 0x5be5, stomp.cu:707)."""

    num_timesteps: int = 51
    num_iterations: int = 20
    num_iterations_after_valid: int = 3
    num_rollouts_new: int = 30
    num_rollouts_old: int = 20
    delta_t: float = 0.1
    control_cost_weight: float = 0.1
    collision_cost_weight: float = 20.0
    exponentiated_cost_sensitivity: float = 2.0
    world_collision_margin: float = 0.02
    self_collision_margin: float = 0.01
    convergence_eps: float = 1.0e-4
    noise_scale: float = 1.0
    collision_check_step: float = 0.05
    collision_margin: float = 0.0
    time_limit_ms: float = 4000.0
    include_self: bool = True
    check_self: bool = True
    seed: int = 0x5BE5

    def to_c(self) -> _lib.StompParams:
        p = _lib.StompParams()
        p.num_iterations = int(self.num_iterations)
        p.num_iterations_after_valid = int(self.num_iterations_after_valid)
        p.num_rollouts_new = int(self.num_rollouts_new)
        p.num_rollouts_old = int(self.num_rollouts_old)
        p.delta_t = float(self.delta_t)
        p.control_cost_weight = float(self.control_cost_weight)
        p.collision_cost_weight = float(self.collision_cost_weight)
        p.exponentiated_cost_sensitivity = float(self.exponentiated_cost_sensitivity)
        p.world_margin = float(self.world_collision_margin)
        p.self_margin = float(self.self_collision_margin)
        p.convergence_eps = float(self.convergence_eps)
        p.noise_scale = float(self.noise_scale)
        p.collision_check_step = float(self.collision_check_step)
        p.collision_margin = float(self.collision_margin)
        p.include_self = int(bool(self.include_self))
        p.check_self = int(bool(self.check_self))
        p.time_limit_ms = float(self.time_limit_ms)
        p.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        return p


def stomp_workspace(robot: RobotModelBuilder, B: int, T: int, settings: Optional[StompSettings] = None,
                    device="cuda"):
    torch = _torch()
    p = (settings or StompSettings()).to_c()
    nbytes = int(_lib.load().ps_stomp_workspace_bytes(_model(robot), int(B), int(T), C.byref(p)))
    if nbytes == 0:
        raise ValueError("invalid STOMP sizes")
    return torch.empty(nbytes, dtype=torch.uint8, device=device)


def stomp_layout(robot: RobotModelBuilder, B: int, T: int, settings: Optional[StompSettings] = None):
    """Byte offsets of the last iteration's rollouts inside the workspace
    (ps_stomp_workspace_layout), as a dict."""
    p = (settings or StompSettings()).to_c()
    lay = _lib.StompLayout()
    _lib.check(_lib.load().ps_stomp_workspace_layout(_model(robot), int(B), int(T), C.byref(p), C.byref(lay)))
    return {"rows": lay.rows, "rollouts": tuple(lay.rollouts), "noise": lay.noise,
            "state_cost": tuple(lay.state_cost), "row_total": tuple(lay.row_total),
            "reuse_index": lay.reuse_index}


def stomp_optimize(robot: RobotModelBuilder, scene, theta, settings: Optional[StompSettings] = None,
                   workspace=None, stream=None) -> ChompResult:
    """Run STOMP on B trajectories ``theta`` [B, T, D] at once (the reference
    runs one, stomp.cu:565-965). ``theta`` is updated in place when it is a
    contiguous float32 CUDA tensor. Synchronises the stream every 8
    iterations. Returns the CHOMPResult-like fields of STOMPResult."""
    torch = _torch()
    settings = settings or StompSettings()
    th = _dev_f32(theta)
    if th.dim() != 3 or th.shape[2] != robot.n_dof:
        raise ValueError("theta must be [B, T, n_dof]")
    B, T, D = th.shape
    best = torch.empty_like(th)
    solved = torch.empty(B, dtype=torch.uint8, device=th.device)
    iters = torch.empty(B, dtype=torch.int32, device=th.device)
    cost = torch.empty(B, dtype=torch.float32, device=th.device)
    p = settings.to_c()
    if workspace is None:
        nbytes = int(_lib.load().ps_stomp_workspace_bytes(_model(robot), B, T, C.byref(p)))
        workspace = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=th.device)
    v = _view(scene)
    _lib.check(_lib.load().ps_stomp_optimize(_model(robot), C.byref(v), th.data_ptr(), B, T, C.byref(p),
                                             best.data_ptr(), solved.data_ptr(), iters.data_ptr(),
                                             cost.data_ptr(), workspace.data_ptr(), workspace.numel(),
                                             _stream(stream)))
    return ChompResult(best, solved.bool(), iters, cost, th)


def stomp_solve(robot: RobotModelBuilder, scene, starts, goals, settings: Optional[StompSettings] = None,
                stream=None, workspace=None) -> ChompResult:
    """STOMP::solve_runtime_scene for B (start, goal) pairs: straight-line
    initialisation (stomp.cu:60-74), the optimiser loop, and the path's first
    and last waypoints set to start and goal (stomp.cu:897-904)."""
    settings = settings or StompSettings()
    theta = chomp_linear_init(robot, starts, goals, settings.num_timesteps)
    res = stomp_optimize(robot, scene, theta, settings, workspace=workspace, stream=stream)
    res.path[:, 0, :] = _dev_f32(starts, robot.n_dof).reshape(-1, robot.n_dof)
    res.path[:, -1, :] = _dev_f32(goals, robot.n_dof).reshape(-1, robot.n_dof)
    return res


# ---------------------------------------------------------------------------
# mixed-request batches
# ---------------------------------------------------------------------------
class MixedBatch:
    """Many edge-check requests and trajectory cost/gradient requests in one
    CUDA-graph launch (ps_batch_*). Results equal ``check_edges`` and
    ``traj_cost`` per request bit for bit. Requests keep references to their
    tensors until ``clear``; ``launch`` is asynchronous on the stream."""

    def __init__(self, robot: RobotModelBuilder, max_edge_requests: int = 0, max_edges: int = 0,
                 max_traj_requests: int = 0, max_waypoints: int = 0, max_traj_len: int = 0):
        self.robot = robot
        lim = _lib.BatchLimits(int(max_edge_requests), int(max_edges), int(max_traj_requests),
                               int(max_waypoints), int(max_traj_len))
        h = C.c_void_p()
        _lib.check(_lib.load().ps_batch_create(_model(robot), C.byref(lim), C.byref(h)))
        self._h = h
        self._keep = []

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("batch is closed")
        return self._h

    def clear(self):
        _lib.check(_lib.load().ps_batch_clear(self.handle))
        self._keep = []

    def add_edges(self, frm, to, samples=None):
        """Queue edges frm/to [n, n_dof]; returns (valid uint8 [n], cost f32 [n])
        filled by the next launch."""
        torch = _torch()
        frm = _dev_f32(frm, self.robot.n_dof)
        to = _dev_f32(to, self.robot.n_dof)
        n = frm.shape[0]
        if to.shape[0] != n:
            raise ValueError("from/to row counts differ")
        if samples is not None:
            samples = torch.as_tensor(samples).to(device=frm.device, dtype=torch.int32).contiguous()
            if samples.shape[0] != n:
                raise ValueError("samples must have one entry per edge")
        valid = torch.empty(n, dtype=torch.uint8, device=frm.device)
        cost = torch.empty(n, dtype=torch.float32, device=frm.device)
        _lib.check(_lib.load().ps_batch_add_edges(self.handle, frm.data_ptr(), to.data_ptr(),
                                                  samples.data_ptr() if samples is not None else None, n,
                                                  valid.data_ptr(), cost.data_ptr()))
        self._keep += [frm, to, samples, valid, cost]
        return valid, cost

    def add_trajectory(self, q, want_waypoint: bool = True, want_traj: bool = True, want_grad: bool = True):
        """Queue one trajectory q [T, n_dof]; returns (waypoint_cost [T] | None,
        traj_cost [1] | None, grad [T, n_dof] | None) filled by the next launch."""
        torch = _torch()
        q = _dev_f32(q, self.robot.n_dof)
        if q.dim() != 2:
            raise ValueError("q must be [T, n_dof]")
        T = q.shape[0]
        wp = torch.empty(T, dtype=torch.float32, device=q.device) if want_waypoint else None
        tc = torch.empty(1, dtype=torch.float32, device=q.device) if want_traj else None
        g = torch.empty_like(q) if want_grad else None
        ptr = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
        _lib.check(_lib.load().ps_batch_add_trajectory(self.handle, q.data_ptr(), T, ptr(wp), ptr(tc), ptr(g)))
        self._keep += [q, wp, tc, g]
        return wp, tc, g

    def add_rollouts(self, rollouts, broadcast_d: bool = False):
        """Queue STOMP rollouts [R, n_dof, T] (the reference layout); returns
        their state costs, [R, T] or [R, n_dof, T] when broadcast_d, filled by
        the next launch (equal to ``rollout_costs`` bit for bit)."""
        torch = _torch()
        r = _dev_f32(rollouts)
        if r.dim() != 3 or r.shape[1] != self.robot.n_dof:
            raise ValueError("rollouts must be [R, n_dof, T]")
        R, D, T = r.shape
        out = torch.empty((R, D, T) if broadcast_d else (R, T), dtype=torch.float32, device=r.device)
        _lib.check(_lib.load().ps_batch_add_rollouts(self.handle, r.data_ptr(), R, T, 1 if broadcast_d else 0,
                                                     out.data_ptr()))
        self._keep += [r, out]
        return out

    def launch(self, scene, edge_params: Optional[EdgeEvalParams] = None,
               cost_params: Optional[CostParams] = None, stream=None):
        ep = (edge_params or EdgeEvalParams()).to_c()
        cp = (cost_params or CostParams()).to_c(_lib.PS_LAYOUT_BTD)
        v = _view(scene)
        _lib.check(_lib.load().ps_batch_launch(self.handle, C.byref(v), C.byref(ep), C.byref(cp),
                                               _stream(stream)))

    def status(self) -> int:
        """PS_OK or PS_ETIMEOUT for the last launch (waits for it)."""
        st = C.c_int(0)
        _lib.check(_lib.load().ps_batch_status(self.handle, C.byref(st)))
        return st.value

    def tune(self, scene, edge_params: Optional[EdgeEvalParams] = None,
             cost_params: Optional[CostParams] = None) -> dict:
        """Autotune the launch shape on the queued requests: the one
        work-queue kernel (128 or 256 threads per block) against the edge
        queue and waypoint kernel side by side (SM shares, block width).
        Returns the chosen shape; later launches use it."""
        ep = (edge_params or EdgeEvalParams()).to_c()
        cp = (cost_params or CostParams()).to_c(_lib.PS_LAYOUT_BTD)
        v = _view(scene)
        t = _lib.BatchTuning()
        _lib.check(_lib.load().ps_batch_tune(self.handle, C.byref(v), C.byref(ep), C.byref(cp), C.byref(t)))
        return {name: getattr(t, name) for name, _ in t._fields_}

    def set_shape(self, layout: int = 0, work_threads: int = 256, work_cost_warps: Optional[int] = None,
                  edge_share: float = 1.0, traj_share: float = 0.5, traj_threads: int = 256) -> None:
        """Launch shape for the next launches: layout 1 = one work-queue
        kernel for edge chunks and waypoint groups (work_cost_warps of its
        warps per block also take waypoint groups; default all); 0 = the
        persistent edge queue and the waypoint kernel side by side. Results
        do not depend on it."""
        t = _lib.BatchTuning()
        t.edge_share, t.traj_share, t.traj_threads, t.traj_tile = edge_share, traj_share, traj_threads, 1
        t.layout, t.work_threads = layout, work_threads
        t.work_cost_warps = work_threads // 32 if work_cost_warps is None else work_cost_warps
        _lib.check(_lib.load().ps_batch_set_shape(self.handle, C.byref(t)))

    def close(self):
        if self._h is not None:
            _lib.check(_lib.load().ps_batch_destroy(self._h))
            self._h = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _make_autograd():
    torch = _torch()
    from torch.autograd.function import once_differentiable

    class _TrajCost(torch.autograd.Function):
        """traj_cost[b] = sum_t w*hinge(q[b,t]) + lambda*sum_d q_d^T R q_d.

        Forward evaluates the cost only (the kernel without the adjoint).
        Backward runs the fused FK + hinge + adjoint kernel on the saved
        configurations: the link transforms are recomputed there rather than
        kept from the forward pass, so nothing per link or per sphere is stored
        between the passes. The scene's device arrays must stay alive until
        backward. First order only: the adjoint is not itself differentiable
        (double backward raises)."""

        @staticmethod
        def forward(ctx, q, robot, scene, params):
            _, tc, _ = traj_cost(robot, scene, q.detach(), params, want_grad=False, want_waypoint=False)
            ctx.save_for_backward(q)
            ctx.robot, ctx.scene, ctx.params = robot, scene, params
            return tc

        @staticmethod
        @once_differentiable
        def backward(ctx, grad_out):
            (q,) = ctx.saved_tensors
            _, _, g = traj_cost(ctx.robot, ctx.scene, q.detach(), ctx.params, want_grad=True, want_waypoint=False)
            return grad_out.reshape(-1, 1, 1) * g, None, None, None

    return _TrajCost


def hinge_cost(q, robot: RobotModelBuilder, scene, params: Optional[CostParams] = None):
    """Differentiable trajectory cost [B] of q [B, T, n_dof]."""
    global _TRAJ_COST
    if _TRAJ_COST is None:
        _TRAJ_COST = _make_autograd()
    return _TRAJ_COST.apply(q, robot, scene, params or CostParams())


_TRAJ_COST = None
