"""Obstacle world: mirrors of ``prrtc.SceneCollisionDataBuilder`` and the
Python ``PlanningScene``.

The device layout is SceneCollisionData's
(code/gpu_planning/cpp/src/collision/scene_collision_data.hh:10-47):
``obb_dims[i] = [dx, dy, dz, 0]`` full extents, ``obb_pose[i] =
[tx, ty, tz, qw, qx, qy, qz, 0]`` the INVERSE pose (world -> box), so that
``p_local = R(q) p_world + t``. The inverse-pose packing restates
code/gpu_planning/python/gpu_planning/substrate/planning_scene.py:40-63.
"""
from __future__ import annotations

import threading
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib


def quat_rotate(q_wxyz: np.ndarray, v: np.ndarray) -> np.ndarray:
    """v + 2w(u x v) + 2u x (u x v) (planning_scene.py:40-51)."""
    w = q_wxyz[0]
    u = np.asarray(q_wxyz[1:], dtype=np.float64)
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def inverse_pose(position, quat_wxyz) -> Tuple[np.ndarray, np.ndarray]:
    """Stored pose of a box placed at ``position`` with orientation
    ``quat_wxyz`` (local -> world): q_stored = conj(Q), t = -R(q_stored) P
    (planning_scene.py:54-63)."""
    q = np.asarray(quat_wxyz, dtype=np.float64)
    q_conj = np.array([q[0], -q[1], -q[2], -q[3]], dtype=np.float64)
    t = -quat_rotate(q_conj, np.asarray(position, dtype=np.float64))
    return t, q_conj


def pack_obbs(dims: np.ndarray, positions: np.ndarray, quats_wxyz: np.ndarray):
    """Host float32 arrays (dims[n,4], pose[n,8], enable[n]) from box
    full extents, world positions and unit quaternions (w,x,y,z)
    (planning_scene.py:189-217)."""
    n = len(dims)
    d = np.zeros((n, 4), np.float32)
    p = np.zeros((n, 8), np.float32)
    en = np.ones((n,), np.uint8)
    for i in range(n):
        d[i, :3] = dims[i]
        qn = np.asarray(quats_wxyz[i], np.float64)
        nrm = np.linalg.norm(qn)
        if nrm > 0:
            qn = qn / nrm
        t, qs = inverse_pose(positions[i], qn)
        p[i, :3] = t
        p[i, 3:7] = qs
    return d, p, en


class SceneCollisionDataBuilder:
    """Drop-in for ``prrtc.SceneCollisionDataBuilder`` (bindings.cpp:363-402).

    Holds raw int64 device pointers (``tensor.data_ptr()``) plus counts and is
    non-owning: the caller keeps the tensors alive while a call uses them.
    ``esdf_mode`` selects the reference nearest-voxel lookup (0) or trilinear
    sampling (1).
    """

    _PTRS = ("obb_dims_ptr", "obb_pose_ptr", "obb_enable_ptr", "voxel_params_ptr",
             "voxel_pose_ptr", "voxel_enable_ptr", "voxel_features_ptr",
             "sphere_acm_mask_ptr", "sphere_obb_acm_mask_ptr",
             "sphere_obb_acm_mask_approx_ptr")

    def __init__(self):
        for p in self._PTRS:
            setattr(self, p, 0)
        self.n_obbs = 0
        self.n_voxel_layers = 0
        self.max_voxels_per_layer = 0
        self.esdf_mode = _lib.PS_ESDF_NEAREST

    def build(self) -> _lib.SceneView:
        v = _lib.SceneView()
        v.obb_dims = self.obb_dims_ptr or None
        v.obb_pose = self.obb_pose_ptr or None
        v.obb_enable = self.obb_enable_ptr or None
        v.n_obbs = int(self.n_obbs)
        v.voxel_params = self.voxel_params_ptr or None
        v.voxel_pose = self.voxel_pose_ptr or None
        v.voxel_enable = self.voxel_enable_ptr or None
        v.voxel_features = self.voxel_features_ptr or None
        v.n_voxel_layers = int(self.n_voxel_layers)
        v.max_voxels_per_layer = int(self.max_voxels_per_layer)
        v.sphere_acm_mask = self.sphere_acm_mask_ptr or None
        v.sphere_obb_acm_mask = self.sphere_obb_acm_mask_ptr or None
        v.sphere_obb_acm_mask_approx = self.sphere_obb_acm_mask_approx_ptr or None
        v.esdf_mode = int(self.esdf_mode)
        return v


class SceneTensors:
    """Device tensors of one scene plus the builder that points at them.

    ``host`` keeps the float32 host arrays (what the oracle consumes).

    Optional allowed-collision masks, uint8 with 0 = pair ignored, indexed by
    the robot descriptor's sphere order (scene_collision_data.hh):
    ``sphere_acm_mask`` [n_spheres, n_voxel_layers], ``sphere_obb_acm_mask``
    [n_spheres, n_obbs] and ``sphere_obb_acm_mask_approx`` [n_approx_spheres,
    n_obbs]. The reference's approximate pass looks neither mask up
    (scene_collision.cuh:584-606 passes sphere index -1), so the approximate
    one is carried for layout parity and changes no result."""

    _MASKS = ("sphere_acm_mask", "sphere_obb_acm_mask", "sphere_obb_acm_mask_approx")

    def __init__(self, obb_dims, obb_pose, obb_enable, voxel_params=None, voxel_pose=None,
                 voxel_enable=None, voxel_features=None, esdf_mode=_lib.PS_ESDF_NEAREST,
                 device="cuda", sphere_acm_mask=None, sphere_obb_acm_mask=None,
                 sphere_obb_acm_mask_approx=None):
        import torch

        self.host = {
            "obb_dims": np.ascontiguousarray(obb_dims, np.float32).reshape(-1, 4),
            "obb_pose": np.ascontiguousarray(obb_pose, np.float32).reshape(-1, 8),
            "obb_enable": np.ascontiguousarray(obb_enable, np.uint8).reshape(-1),
        }
        n_layers = 0 if voxel_params is None else int(np.asarray(voxel_params).reshape(-1, 4).shape[0])
        if n_layers:
            self.host["voxel_params"] = np.ascontiguousarray(voxel_params, np.float32).reshape(-1, 4)
            self.host["voxel_pose"] = np.ascontiguousarray(voxel_pose, np.float32).reshape(-1, 8)
            self.host["voxel_enable"] = (np.ones(n_layers, np.uint8) if voxel_enable is None
                                         else np.ascontiguousarray(voxel_enable, np.uint8).reshape(-1))
            self.host["voxel_features"] = np.ascontiguousarray(voxel_features, np.float32).reshape(n_layers, -1)
        n_obbs = self.host["obb_dims"].shape[0]
        for name, m, cols in zip(self._MASKS, (sphere_acm_mask, sphere_obb_acm_mask, sphere_obb_acm_mask_approx),
                                 (n_layers, n_obbs, n_obbs)):
            if m is None:
                continue
            m = np.ascontiguousarray(m, np.uint8)
            if cols == 0 or m.size % cols:
                raise ValueError(f"{name}: {m.size} entries is not a whole number of rows of {cols}")
            self.host[name] = m.reshape(-1, cols)
        self.esdf_mode = esdf_mode
        self.device = device
        dev = torch.device(device)
        self.tensors = {k: torch.from_numpy(v.copy()).to(dev) for k, v in self.host.items()}
        b = SceneCollisionDataBuilder()
        t = self.tensors
        b.n_obbs = self.host["obb_dims"].shape[0]
        if b.n_obbs:
            b.obb_dims_ptr = t["obb_dims"].data_ptr()
            b.obb_pose_ptr = t["obb_pose"].data_ptr()
            b.obb_enable_ptr = t["obb_enable"].data_ptr()
        if n_layers:
            b.voxel_params_ptr = t["voxel_params"].data_ptr()
            b.voxel_pose_ptr = t["voxel_pose"].data_ptr()
            b.voxel_enable_ptr = t["voxel_enable"].data_ptr()
            b.voxel_features_ptr = t["voxel_features"].data_ptr()
            b.n_voxel_layers = n_layers
            b.max_voxels_per_layer = self.host["voxel_features"].shape[1]
        for name in self._MASKS:
            if name in t:
                setattr(b, name + "_ptr", t[name].data_ptr())
        b.esdf_mode = esdf_mode
        self.builder = b

    @property
    def masks(self) -> Dict[str, np.ndarray]:
        """The host masks by the oracle's names (acm, obb_acm, obb_acm_apx)."""
        keys = dict(zip(self._MASKS, ("acm", "obb_acm", "obb_acm_apx")))
        return {keys[k]: self.host[k] for k in self._MASKS if k in self.host}

    @property
    def n_obbs(self) -> int:
        return self.host["obb_dims"].shape[0]

    def view(self) -> _lib.SceneView:
        return self.builder.build()


class PlanningScene:
    """OBB collision world (planning_scene.py:66-242): named cuboids kept on
    the host, packed into device tensors on demand."""

    def __init__(self, num_joints: int = 0, robot_id: str = "robot", device: str = "cuda"):
        self._num_joints = int(num_joints)
        self._robot_id = robot_id
        self._device = device
        self._cuboids: Dict[str, Tuple[np.ndarray, np.ndarray, np.ndarray]] = {}
        self._voxel_plan_lock = threading.RLock()
        self._dirty = True
        self._tensors: Optional[SceneTensors] = None

    @classmethod
    def from_robot_asset(cls, asset_path, device: str = "cuda") -> "PlanningScene":
        """A scene sized to a robot YAML asset: its name and n_dof
        (planning_scene.py:92-100)."""
        from .robot import load_robot_asset

        asset = load_robot_asset(asset_path)
        return cls(num_joints=asset["n_dof"], robot_id=asset["name"], device=device)

    @property
    def num_joints(self) -> int:
        return self._num_joints

    @property
    def robot_id(self) -> str:
        return self._robot_id

    @property
    def n_obbs(self) -> int:
        """Boxes in the last built collision data (planning_scene.py:111-113,
        set when the tensors are rebuilt)."""
        return 0 if self._tensors is None else self._tensors.n_obbs

    @property
    def current_obstacles(self) -> List[Dict[str, Any]]:
        """The cuboids as update_world takes them (planning_scene.py:115-128):
        name, type, dims, position, quaternion (w, x, y, z)."""
        return [{"name": name, "type": "cuboid", "dims": d.tolist(), "position": p.tolist(),
                 "quaternion": q.tolist()} for name, (d, p, q) in self._cuboids.items()]

    def add_cuboid(self, name: str, dims: Sequence[float], position: Sequence[float],
                   quaternion=(1.0, 0.0, 0.0, 0.0)) -> None:
        q = np.asarray(quaternion, np.float64).reshape(4)
        n = np.linalg.norm(q)
        if n > 0:
            q = q / n
        with self._voxel_plan_lock:
            self._cuboids[name] = (np.asarray(dims, np.float64).reshape(3),
                                   np.asarray(position, np.float64).reshape(3), q)
            self._dirty = True

    def remove_cuboid(self, name: str) -> bool:
        with self._voxel_plan_lock:
            existed = self._cuboids.pop(name, None) is not None
            self._dirty |= existed
            return existed

    def clear(self) -> None:
        with self._voxel_plan_lock:
            if self._cuboids:
                self._cuboids.clear()
                self._dirty = True

    def update_world(self, obstacles: List[Dict[str, Any]]) -> None:
        with self._voxel_plan_lock:
            self._cuboids.clear()
            for i, obs in enumerate(obstacles):
                name = obs.get("name", f"obs_{i}")
                if "pose" in obs:
                    pos, quat = obs["pose"][0:3], obs["pose"][3:7]
                else:
                    pos, quat = obs["position"], obs.get("quaternion", (1.0, 0.0, 0.0, 0.0))
                self.add_cuboid(name, obs["dims"], pos, quat)
            self._dirty = True

    def build_scene_collision_data(self) -> Optional[SceneCollisionDataBuilder]:
        """Filled builder, or None for an empty world (planning_scene.py:219-242).
        Hold ``_voxel_plan_lock`` while the returned pointers are in use."""
        if self._dirty:
            if not self._cuboids:
                self._tensors = None
            else:
                vals = list(self._cuboids.values())
                d, p, en = pack_obbs(np.stack([v[0] for v in vals]), np.stack([v[1] for v in vals]),
                                     np.stack([v[2] for v in vals]))
                self._tensors = SceneTensors(d, p, en, device=self._device)
            self._dirty = False
        return None if self._tensors is None else self._tensors.builder
