"""Robot model: host mirror of ``prrtc.RobotModelBuilder`` over the C ABI.

Field names, defaults and methods follow the reference builder
(code/gpu_planning/cpp/src/python/bindings.cpp:118-225): writable flat lists,
a lazy idempotent ``build()`` that owns the device upload,
``update_joint_limits()`` and ``destroy()``. The YAML asset loader and the
approximate-sphere derivation restate
code/gpu_planning/python/gpu_planning/substrate/robot_model_loader.py:32-190.
"""
from __future__ import annotations

import ctypes as C
from collections import defaultdict
from pathlib import Path
from typing import Any, Dict, List, Sequence

import numpy as np

from . import _lib


def _arr(values, dtype):
    return np.ascontiguousarray(np.asarray(values, dtype=dtype).reshape(-1))


def build_approx_spheres(spheres_flat: Sequence[float], sphere_to_joint: Sequence[int],
                         n_joints: int):
    """One bounding sphere per joint: centroid of the joint's spheres, radius
    max(|c - a_i| + r_i) (robot_model_loader.py:32-64). Spheres with r <= 0 are
    ignored; joints without spheres get none. Arithmetic in Python floats
    (FP64), the same sums in the same order as the reference."""
    joint_spheres: Dict[int, list] = defaultdict(list)
    n = len(sphere_to_joint)
    for si in range(n):
        x, y, z, r = (float(spheres_flat[si * 4 + k]) for k in range(4))
        if r <= 0.0:
            continue
        joint_spheres[int(sphere_to_joint[si])].append((x, y, z, r))
    flat: List[float] = []
    joints: List[int] = []
    for j in range(n_joints):
        lst = joint_spheres.get(j, [])
        if not lst:
            continue
        cx = sum(s[0] for s in lst) / len(lst)
        cy = sum(s[1] for s in lst) / len(lst)
        cz = sum(s[2] for s in lst) / len(lst)
        max_r = 0.0
        for x, y, z, r in lst:
            max_r = max(max_r, ((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) ** 0.5 + r)
        flat.extend([cx, cy, cz, max_r])
        joints.append(j)
    return flat, joints


def build_approx_self_cc_ranges(full_ranges: Sequence[int], sphere_to_joint: Sequence[int],
                                approx_sphere_to_joint: Sequence[int]):
    """Joint-level approximate self-collision ranges covering every joint pair
    of the full ranges (robot_model_loader.py:67-115). Flat, end inclusive."""
    if len(full_ranges) == 0:
        return []
    joint_to_approx = {int(j): ai for ai, j in enumerate(approx_sphere_to_joint)}
    pairs: Dict[int, set] = defaultdict(set)
    for e in range(len(full_ranges) // 3):
        si, start, end = (int(full_ranges[e * 3 + k]) for k in range(3))
        ji = int(sphere_to_joint[si])
        for sj in range(start, end + 1):
            jj = int(sphere_to_joint[sj])
            if ji == jj:
                continue
            ai, aj = joint_to_approx.get(ji), joint_to_approx.get(jj)
            if ai is None or aj is None:
                continue
            pairs[ai].add(aj)
            pairs[aj].add(ai)
    out: List[int] = []
    for ai in sorted(pairs):
        partners = sorted(p for p in pairs[ai] if p > ai)
        if not partners:
            continue
        lo = hi = partners[0]
        for p in partners[1:]:
            if p == hi + 1:
                hi = p
            else:
                out.extend([ai, lo, hi])
                lo = hi = p
        out.extend([ai, lo, hi])
    return out


def load_robot_asset(path) -> Dict[str, Any]:
    """Parse a robot YAML asset into flat host arrays plus the derived
    approximate model (robot_model_loader.py:118-190)."""
    import yaml

    with open(Path(path), "r") as f:
        doc = yaml.safe_load(f)
    n_dof, n_joints = int(doc["n_dof"]), int(doc["n_joints"])
    ft = [float(v) for row in doc["fixed_transforms"] for v in row]
    if len(ft) != n_joints * 16:
        raise ValueError(f"fixed_transforms has {len(ft)} values, expected {n_joints * 16}")
    spheres = [float(v) for s in doc["spheres"] for v in s]
    s2j = [int(v) for v in doc["sphere_to_joint"]]
    if len(spheres) != len(s2j) * 4:
        raise ValueError("spheres / sphere_to_joint size mismatch")
    ranges = [int(v) for c in doc["self_cc_ranges"] for v in c]
    asset = {
        "name": doc.get("name", "robot"),
        "n_dof": n_dof,
        "n_joints": n_joints,
        "joint_types": [int(v) for v in doc["joint_types"]],
        "fixed_transforms": ft,
        "spheres_flat": spheres,
        "sphere_to_joint": s2j,
        "self_cc_ranges_flat": ranges,
        "joint_lower": [float(v) for v in doc["joint_lower"]],
        "joint_upper": [float(v) for v in doc["joint_upper"]],
        "joint_parents": [int(v) for v in doc.get("joint_parents", [max(i - 1, 0) for i in range(n_joints)])],
        "joint_id_to_dof": [int(v) for v in doc.get("joint_id_to_dof", [i - 1 for i in range(n_joints)])],
        "t_memory_idx": [int(v) for v in doc.get("t_memory_idx", [0] + [1] * (n_joints - 1))],
        "dfs_order": [int(v) for v in doc.get("dfs_order", list(range(n_joints)))],
    }
    for k in ("joint_parents", "joint_id_to_dof", "t_memory_idx", "dfs_order"):
        if len(asset[k]) != n_joints:
            raise ValueError(f"{k} has {len(asset[k])} entries, expected {n_joints}")
    asset["n_t_slots"] = max(asset["t_memory_idx"]) + 1
    complete_approx_model(asset)
    return asset


def complete_approx_model(asset: Dict[str, Any]) -> Dict[str, Any]:
    """Fill approx_* fields from the full model when absent."""
    if not asset.get("approx_sphere_to_joint"):
        a_flat, a_j = build_approx_spheres(asset["spheres_flat"], asset["sphere_to_joint"],
                                           asset["n_joints"])
        asset["approx_spheres_flat"] = a_flat
        asset["approx_sphere_to_joint"] = a_j
    if "approx_self_cc_ranges_flat" not in asset:
        asset["approx_self_cc_ranges_flat"] = build_approx_self_cc_ranges(
            asset["self_cc_ranges_flat"], asset["sphere_to_joint"], asset["approx_sphere_to_joint"])
    return asset


_BUILDER_FIELDS = (
    "fixed_transforms", "joint_types", "spheres_flat", "sphere_to_joint", "self_cc_ranges_flat",
    "approx_spheres_flat", "approx_sphere_to_joint", "approx_self_cc_ranges_flat",
    "approx_fixed_transforms", "approx_joint_types", "joint_lower", "joint_upper",
    "joint_parents", "joint_id_to_dof", "t_memory_idx", "dfs_order",
)


class RobotModelBuilder:
    """Drop-in for ``prrtc.RobotModelBuilder`` (bindings.cpp:118-225, 960-989).

    Set the flat fields, then ``build()`` (lazy, idempotent) uploads the model
    to the current CUDA device through ``ps_model_create``. The builder owns
    the device model; ``destroy()`` or garbage collection frees it.
    """

    # Mesh BVH fields of the reference builder (bindings.cpp:980-984). Mesh
    # collision is outside this substrate: the fields are accepted so that
    # assets and callers that set them keep working, but they are not uploaded
    # and any request for mesh checks (EdgeEvalParams.enable_mesh) is refused.
    MESH_FIELDS = ("mesh_bvh_nodes", "mesh_tri_vertices", "mesh_link_bvh_root", "mesh_link_tri_offset",
                   "mesh_link_tri_count")

    def __init__(self):
        self.n_dof = 0
        self.n_joints = 0
        for f in _BUILDER_FIELDS + self.MESH_FIELDS:
            setattr(self, f, [])
        self._handle = None

    # -- construction helpers ------------------------------------------------
    @classmethod
    def from_asset(cls, asset: Dict[str, Any]) -> "RobotModelBuilder":
        b = cls()
        b.n_dof = int(asset["n_dof"])
        b.n_joints = int(asset["n_joints"])
        for f in _BUILDER_FIELDS:
            if f in asset and asset[f] is not None:
                setattr(b, f, list(asset[f]))
        return b

    def descriptor(self):
        """(ModelDesc, keepalive) with numpy-backed host arrays."""
        keep = []

        def fptr(values):
            if values is None or len(values) == 0:
                return None
            a = _arr(values, np.float32)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_float))

        def iptr(values):
            if values is None or len(values) == 0:
                return None
            a = _arr(values, np.int32)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_int))

        d = _lib.ModelDesc()
        d.n_dof, d.n_joints = int(self.n_dof), int(self.n_joints)
        d.fixed_transforms = fptr(self.fixed_transforms)
        d.joint_types = iptr(self.joint_types)
        d.n_spheres = len(self.sphere_to_joint)
        d.spheres = fptr(self.spheres_flat)
        d.sphere_to_joint = iptr(self.sphere_to_joint)
        d.n_self_cc_ranges = len(self.self_cc_ranges_flat) // 3
        d.self_cc_ranges = iptr(self.self_cc_ranges_flat)
        d.n_approx_spheres = len(self.approx_sphere_to_joint)
        d.approx_spheres = fptr(self.approx_spheres_flat)
        d.approx_sphere_to_joint = iptr(self.approx_sphere_to_joint)
        d.n_approx_self_cc_ranges = len(self.approx_self_cc_ranges_flat) // 3
        d.approx_self_cc_ranges = iptr(self.approx_self_cc_ranges_flat)
        d.approx_fixed_transforms = fptr(self.approx_fixed_transforms)
        d.approx_joint_types = iptr(self.approx_joint_types)
        d.joint_lower = fptr(self.joint_lower)
        d.joint_upper = fptr(self.joint_upper)
        d.joint_parents = iptr(self.joint_parents)
        d.joint_id_to_dof = iptr(self.joint_id_to_dof)
        d.t_memory_idx = iptr(self.t_memory_idx)
        d.dfs_order = iptr(self.dfs_order)
        return d, keep

    # -- reference API ---------------------------------------------------------
    def build(self):
        """Upload to the device once (bindings.cpp:157-179). Returns self."""
        if self._handle is None:
            lib = _lib.load()
            d, keep = self.descriptor()
            h = C.c_void_p()
            _lib.check(lib.ps_model_create(C.byref(d), C.byref(h)))
            self._handle = h
        return self

    build_on_device = build

    @property
    def built(self) -> bool:
        return self._handle is not None

    @property
    def handle(self) -> C.c_void_p:
        return self.build()._handle

    def update_joint_limits(self):
        """Re-upload joint limits without a rebuild (bindings.cpp:181-205)."""
        if self._handle is None:
            self.build()
            return
        if len(self.joint_lower) != self.n_dof or len(self.joint_upper) != self.n_dof:
            raise RuntimeError("joint_lower/joint_upper size != n_dof")
        lo = _arr(self.joint_lower, np.float32)
        hi = _arr(self.joint_upper, np.float32)
        _lib.check(_lib.load().ps_model_set_limits(
            self._handle, lo.ctypes.data_as(C.POINTER(C.c_float)),
            hi.ctypes.data_as(C.POINTER(C.c_float))))

    def info(self) -> Dict[str, Any]:
        inf = _lib.ModelInfo()
        _lib.check(_lib.load().ps_model_get_info(self.handle, C.byref(inf)))
        return {name: getattr(inf, name) for name, _ in inf._fields_}

    def destroy(self):
        if self._handle is not None:
            lib = _lib.load()
            lib.ps_model_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def build_robot_model(path) -> RobotModelBuilder:
    """Load a YAML asset and return a built builder
    (robot_model_loader.py:193-243)."""
    return RobotModelBuilder.from_asset(load_robot_asset(path)).build()
