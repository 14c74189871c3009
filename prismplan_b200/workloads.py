"""Seeded synthetic workloads with the benchmark shapes.

The reference measures planners on MotionBenchMaker problems; that dataset is
not available here, so these generators stand in for it with fixed seeds
(seed = 1000 + workload index, numpy default_rng):

  1  configs  : Panda-like 7R chain (59 spheres), 16 OBBs, 4096 configurations
  2  edges    : same chain, 64 OBBs, 65,536 edges, L-inf step 0.01 rad (1..600)
  3  chomp    : 256 trajectories x 64 waypoints x 7 DoF, 64 OBBs, eps 0.05
  4  stomp    : Fetch-like 8-DoF (prismatic torso + 7R, 70 spheres), 96 OBBs,
                32 x 128 rollouts x 100 waypoints, noise L z with L from R^-1
  5  mixed    : Baxter-like 14-DoF tree (two 7R arms on one base, ~110
                spheres), 128 OBBs + 128^3 ESDF (5 mm voxels)
"""
from __future__ import annotations

import math
from typing import Dict, List

import numpy as np

from . import _lib
from .robot import build_approx_self_cc_ranges, build_approx_spheres

X_PRISM, Y_PRISM, Z_PRISM, X_ROT, Y_ROT, Z_ROT = range(6)


# ---------------------------------------------------------------------------
# robots
# ---------------------------------------------------------------------------
def _ft(R: np.ndarray, t) -> List[float]:
    M = np.eye(4)
    M[:3, :3] = R
    M[:3, 3] = t
    return [float(v) for v in M.reshape(-1)]


def _rx(a: float) -> np.ndarray:
    c, s = round(math.cos(a), 12), round(math.sin(a), 12)
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]], dtype=np.float64)


def _finish(asset: Dict) -> Dict:
    a_flat, a_j = build_approx_spheres(asset["spheres_flat"], asset["sphere_to_joint"], asset["n_joints"])
    asset["approx_spheres_flat"] = a_flat
    asset["approx_sphere_to_joint"] = a_j
    asset["approx_self_cc_ranges_flat"] = build_approx_self_cc_ranges(
        asset["self_cc_ranges_flat"], asset["sphere_to_joint"], a_j)
    asset["n_t_slots"] = max(asset["t_memory_idx"]) + 1
    return asset


def _arm(rng, n_links: int, counts: List[int], first_joint: int, base_offset, side: float,
         types: List[int]):
    """Fixed transforms and link spheres of one serial arm.

    Link offsets U(0.08, 0.33) m alternate between the joint axis (z) and the
    y axis of the joint frame; frames twist by +-90 deg about x so consecutive
    axes are orthogonal, as on a Panda-type arm."""
    fts, sph, s2j = [], [], []
    offsets = []
    for k in range(n_links):
        d = float(rng.uniform(0.08, 0.33))
        if k == 0:
            t = np.asarray(base_offset, np.float64) + np.array([0.0, 0.0, d])
            R = _rx(0.0)
        else:
            t = np.array([0.0, side * (-d if k % 2 else d), 0.0]) if k % 2 else np.array([0.0, 0.0, d])
            R = _rx(-math.pi / 2 if k % 2 else math.pi / 2)
        fts.append(_ft(R, t))
        offsets.append(t)
    # spheres of link k live in joint k's frame along the segment to joint k+1
    for k in range(n_links):
        nxt = offsets[k + 1] if k + 1 < n_links else np.array([0.0, 0.0, 0.12])
        if k + 1 < n_links:
            # next joint origin expressed in this frame = its translation
            seg = nxt
        else:
            seg = nxt
        for c in range(counts[k]):
            s = (c + 0.5) / counts[k]
            p = s * seg + rng.normal(0.0, 0.015, 3)
            r = float(rng.uniform(0.03, 0.08))
            sph.extend([float(p[0]), float(p[1]), float(p[2]), r])
            s2j.append(first_joint + k)
    return fts, sph, s2j


def _self_ranges(s2j: List[int], parents: List[int]) -> List[int]:
    """{sphere, start, end} ranges pairing each sphere with later spheres on
    joints that are neither itself, its parent nor its child."""
    n = len(s2j)
    out = []
    for i in range(n):
        ji = s2j[i]
        ok = [j for j in range(i + 1, n)
              if s2j[j] != ji and parents[s2j[j]] != ji and parents[ji] != s2j[j]]
        if not ok:
            continue
        lo = hi = ok[0]
        for j in ok[1:]:
            if j == hi + 1:
                hi = j
            else:
                out.extend([i, lo, hi])
                lo = hi = j
        out.extend([i, lo, hi])
    return out


def panda_like(seed: int = 1001, n_spheres: int = 59) -> Dict:
    """7-revolute serial chain, 59 spheres r ~ U(0.03, 0.08) on links 1-7,
    limits +-2.9 rad."""
    rng = np.random.default_rng(seed)
    counts = [n_spheres // 7] * 7
    for k in range(n_spheres - sum(counts)):
        counts[k % 7] += 1
    fts, sph, s2j = _arm(rng, 7, counts, 1, (0.0, 0.0, 0.0), 1.0, [Z_ROT] * 7)
    n_joints = 8
    parents = [0] + list(range(7))
    asset = {
        "name": "panda_like", "n_dof": 7, "n_joints": n_joints,
        "joint_types": [X_ROT] + [Z_ROT] * 7,
        "fixed_transforms": _ft(np.eye(3), (0, 0, 0)) + [v for f in fts for v in f],
        "spheres_flat": sph, "sphere_to_joint": s2j,
        "joint_lower": [-2.9] * 7, "joint_upper": [2.9] * 7,
        "joint_parents": parents, "joint_id_to_dof": [-1] + list(range(7)),
        "t_memory_idx": [0] + [1] * 7, "dfs_order": list(range(8)),
    }
    asset["self_cc_ranges_flat"] = _self_ranges(s2j, parents)
    return _finish(asset)


def fetch_like(seed: int = 1004) -> Dict:
    """Prismatic torso (Z_PRISM, 0..0.386 m) + 7 revolute joints with mixed
    axes, 70 spheres (10 base, 12 torso, 48 arm)."""
    rng = np.random.default_rng(seed)
    types = [X_ROT, Z_PRISM, Z_ROT, Y_ROT, X_ROT, Y_ROT, X_ROT, Y_ROT, X_ROT]
    fts = [_ft(np.eye(3), (0, 0, 0)), _ft(np.eye(3), (-0.086, 0.0, 0.377))]
    sph, s2j = [], []
    for c in range(10):      # base disc
        a = 2 * math.pi * c / 10
        sph.extend([0.22 * math.cos(a), 0.22 * math.sin(a), 0.1, float(rng.uniform(0.05, 0.08))])
        s2j.append(0)
    for c in range(12):      # torso column
        sph.extend([-0.05, 0.0, 0.05 + 0.06 * c, float(rng.uniform(0.05, 0.08))])
        s2j.append(1)
    arm_ft, arm_sph, arm_s2j = _arm(rng, 7, [7, 7, 7, 7, 7, 7, 6], 2, (0.12, 0.0, 0.35), 1.0, types[2:])
    fts += arm_ft
    sph += arm_sph
    s2j += arm_s2j
    parents = [0] + list(range(8))
    asset = {
        "name": "fetch_like", "n_dof": 8, "n_joints": 9, "joint_types": types,
        "fixed_transforms": [v for f in fts for v in f],
        "spheres_flat": sph, "sphere_to_joint": s2j,
        "joint_lower": [0.0] + [-2.9] * 7, "joint_upper": [0.386] + [2.9] * 7,
        "joint_parents": parents, "joint_id_to_dof": [-1] + list(range(8)),
        "t_memory_idx": [0] + [1] * 8, "dfs_order": list(range(9)),
    }
    asset["self_cc_ranges_flat"] = _self_ranges(s2j, parents)
    return _finish(asset)


def baxter_like(seed: int = 1005) -> Dict:
    """Branching tree: two 7R arms hanging off the root (joint 8's parent is
    0), 6 base spheres + 52 per arm = 110 spheres."""
    rng = np.random.default_rng(seed)
    fts = [_ft(np.eye(3), (0, 0, 0))]
    sph, s2j = [], []
    for c in range(6):
        sph.extend([0.0, -0.15 + 0.06 * c, 0.25, float(rng.uniform(0.05, 0.08))])
        s2j.append(0)
    counts = [8, 8, 7, 8, 7, 7, 7]
    a_ft, a_sph, a_s2j = _arm(rng, 7, counts, 1, (0.06, 0.26, 0.35), 1.0, [Z_ROT] * 7)
    b_ft, b_sph, b_s2j = _arm(rng, 7, counts, 8, (0.06, -0.26, 0.35), -1.0, [Z_ROT] * 7)
    fts += a_ft + b_ft
    sph += a_sph + b_sph
    s2j += a_s2j + b_s2j
    parents = [0, 0, 1, 2, 3, 4, 5, 6, 0, 8, 9, 10, 11, 12, 13]
    asset = {
        "name": "baxter_like", "n_dof": 14, "n_joints": 15, "joint_types": [X_ROT] + [Z_ROT] * 14,
        "fixed_transforms": [v for f in fts for v in f],
        "spheres_flat": sph, "sphere_to_joint": s2j,
        "joint_lower": [-2.9] * 14, "joint_upper": [2.9] * 14,
        "joint_parents": parents, "joint_id_to_dof": [-1] + list(range(14)),
        "t_memory_idx": [0] + [1] * 14, "dfs_order": list(range(15)),
    }
    asset["self_cc_ranges_flat"] = _self_ranges(s2j, parents)
    return _finish(asset)


def generic_chain(seed: int = 1006, n_links: int = 7, spheres_per_link: int = 6) -> Dict:
    """Serial chain whose fixed transforms carry generic rotations (uniform
    SO(3)) and mixed joint types (X/Y/Z revolute, one prismatic), so that every
    joint-step column combines two nonzero products."""
    rng = np.random.default_rng(seed)
    types = [X_ROT] + [int(t) for t in rng.choice([X_ROT, Y_ROT, Z_ROT], n_links)]
    types[3] = int(rng.choice([X_PRISM, Y_PRISM, Z_PRISM]))
    fts = [_ft(np.eye(3), (0, 0, 0))]
    sph, s2j = [], []
    for k in range(n_links):
        qv = rng.normal(size=4)
        qv /= np.linalg.norm(qv)
        w, x, y, z = qv
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        t = rng.uniform(-0.25, 0.25, 3) + np.array([0.0, 0.0, 0.12])
        fts.append(_ft(R, t))
        for c in range(spheres_per_link):
            p = rng.uniform(-0.12, 0.12, 3)
            sph.extend([float(p[0]), float(p[1]), float(p[2]), float(rng.uniform(0.03, 0.08))])
            s2j.append(k + 1)
    parents = [0] + list(range(n_links))
    lo = [-2.9] * n_links
    hi = [2.9] * n_links
    lo[2], hi[2] = -0.3, 0.3     # the prismatic joint (types[3] drives dof 2)
    asset = {
        "name": "generic_chain", "n_dof": n_links, "n_joints": n_links + 1, "joint_types": types,
        "fixed_transforms": [float(np.float32(v)) for f in fts for v in f],
        "spheres_flat": sph, "sphere_to_joint": s2j, "joint_lower": lo, "joint_upper": hi,
        "joint_parents": parents, "joint_id_to_dof": [-1] + list(range(n_links)),
        "t_memory_idx": [0] + [1] * n_links, "dfs_order": list(range(n_links + 1)),
    }
    asset["self_cc_ranges_flat"] = _self_ranges(s2j, parents)
    return _finish(asset)


# ---------------------------------------------------------------------------
# scenes
# ---------------------------------------------------------------------------
def random_obbs(rng, n: int, lo=-1.0, hi=1.0, half_lo=0.02, half_hi=0.3):
    """Centres U([lo,hi]^3), half-extents U(half_lo, half_hi), uniform SO(3)
    rotations (normalised Gaussian quaternions). Returns host arrays in the
    SceneCollisionData layout (dims full extents, inverse pose)."""
    from .scene import pack_obbs

    centres = rng.uniform(lo, hi, (n, 3))
    half = rng.uniform(half_lo, half_hi, (n, 3))
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return pack_obbs(2.0 * half, centres, q)


def random_esdf(rng, n_vox: int = 128, voxel: float = 0.005, n_boxes: int = 16,
                centre=(0.45, 0.0, 0.45)):
    """One ESDF layer: n_vox^3 voxels of `voxel` m, signed distance to the union
    of `n_boxes` axis-aligned random boxes, positive inside (penetration
    depth), negative outside, the outermost 2 voxel layers set to the -1000
    unobserved sentinel. Grid-local origin at the grid centre; the stored pose
    is the inverse of a pure translation to `centre`."""
    ext = (n_vox - 1) * voxel
    params = np.array([[ext, ext, ext, voxel]], np.float32)
    pose = np.zeros((1, 8), np.float32)
    pose[0, :3] = -np.asarray(centre, np.float32)
    pose[0, 3] = 1.0
    g = (np.arange(n_vox, dtype=np.float64) + 0.5) * voxel - ext * 0.5
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    P = np.stack([X, Y, Z], -1).reshape(-1, 3)
    best = np.full(P.shape[0], -1e9)
    for _ in range(n_boxes):
        c = rng.uniform(-ext * 0.35, ext * 0.35, 3)
        h = rng.uniform(0.02, 0.08, 3)
        q = np.abs(P - c) - h
        outside = np.linalg.norm(np.maximum(q, 0.0), axis=1)
        inside = np.minimum(q.max(axis=1), 0.0)
        sdf = outside + inside            # standard SDF, negative inside
        best = np.maximum(best, -sdf)     # "positive = inside": max over boxes of -sdf
    F = best.reshape(n_vox, n_vox, n_vox).astype(np.float32)
    F[:2, :, :] = F[-2:, :, :] = -1000.0
    F[:, :2, :] = F[:, -2:, :] = -1000.0
    F[:, :, :2] = F[:, :, -2:] = -1000.0
    return params, pose, np.ones(1, np.uint8), F.reshape(1, -1)


# ---------------------------------------------------------------------------
# queries
# ---------------------------------------------------------------------------
def uniform_configs(rng, asset: Dict, n: int) -> np.ndarray:
    lo = np.asarray(asset["joint_lower"], np.float64)
    hi = np.asarray(asset["joint_upper"], np.float64)
    return (lo + rng.random((n, len(lo))) * (hi - lo)).astype(np.float32)


def free_pairs(rng, asset: Dict, n: int, is_free, oversample: int = 4):
    """n (start, goal) pairs drawn uniformly within the limits from
    configurations that ``is_free`` (a callable, [m, D] -> bool [m]) accepts,
    as a planning benchmark poses them (both endpoints collision-free).
    Raises if fewer than 2 n candidates pass."""
    cand = uniform_configs(rng, asset, max(2 * n * oversample, 2))
    free = cand[np.asarray(is_free(cand), bool)]
    if len(free) < 2 * n:
        raise ValueError(f"only {len(free)} of {len(cand)} candidates are collision-free")
    return free[:n].copy(), free[n:2 * n].copy()


def linf_samples(frm: np.ndarray, to: np.ndarray, step: float, max_samples: int = 600) -> np.ndarray:
    """G_e = clamp(ceil(max_i |to_i - from_i| / step), 1, max_samples), computed
    in float32 as the device does."""
    d = np.abs(to.astype(np.float32) - frm.astype(np.float32)).max(axis=1)
    g = np.ceil(d / np.float32(step)).astype(np.int64)
    return np.clip(g, 1, max_samples).astype(np.int32)


def edge_batch(rng, asset: Dict, n: int, step: float = 0.01, max_samples: int = 600):
    """Half uniform (from, to) pairs, half short local edges to = from +
    U(-0.3, 0.3) clamped to the limits, interleaved. Returns from, to, G."""
    lo = np.asarray(asset["joint_lower"], np.float32)
    hi = np.asarray(asset["joint_upper"], np.float32)
    frm = uniform_configs(rng, asset, n)
    far = uniform_configs(rng, asset, n)
    near = np.clip(frm + rng.uniform(-0.3, 0.3, frm.shape).astype(np.float32), lo, hi)
    to = np.where((np.arange(n) % 2 == 0)[:, None], far, near).astype(np.float32)
    return frm, to, linf_samples(frm, to, step, max_samples)


def straight_trajectories(rng, asset: Dict, B: int, T: int, noise: float = 0.05) -> np.ndarray:
    """[B, T, D] straight lines between random start/goal plus N(0, noise)
    interior noise, endpoints pinned, clamped to the limits."""
    lo = np.asarray(asset["joint_lower"], np.float64)
    hi = np.asarray(asset["joint_upper"], np.float64)
    D = len(lo)
    s = lo + rng.random((B, D)) * (hi - lo)
    g = lo + rng.random((B, D)) * (hi - lo)
    f = np.linspace(0.0, 1.0, T)[None, :, None]
    q = s[:, None, :] * (1 - f) + g[:, None, :] * f
    q[:, 1:-1, :] += rng.normal(0.0, noise, (B, T - 2, D))
    return np.clip(q, lo, hi).astype(np.float32)


def control_cost_R(T: int, dt: float) -> np.ndarray:
    """R = dt A^T A, central T x T block of the 6-padded 5-point acceleration
    operator (chomp_precompute.cpp:20-37), FP64."""
    pad, Np = 6, T + 12
    coeff = np.array([0.0, -1 / 12, 16 / 12, -30 / 12, 16 / 12, -1 / 12, 0.0]) / (dt * dt)
    A = np.zeros((Np, Np))
    for i in range(Np):
        for j in range(-3, 4):
            if 0 <= i + j < Np:
                A[i, i + j] = coeff[j + 3]
    return (dt * (A.T @ A))[pad:pad + T, pad:pad + T]


def stomp_noise_L(T: int, dt: float) -> np.ndarray:
    """Cholesky factor of (R + 1e-8 I)^-1 scaled to max entry 1/T
    (stomp_precompute.cpp:46-68), FP64."""
    R = control_cost_R(T, dt) + 1e-8 * np.eye(T)
    Rinv = np.linalg.inv(R)
    Rinv *= (1.0 / T) / max(Rinv.max(), 1e-12)
    Rinv = 0.5 * (Rinv + Rinv.T)
    return np.linalg.cholesky(Rinv)


def workload(index: int, scale: float = 1.0) -> Dict:
    """The synthetic workload `index` (1..5). `scale` < 1 shrinks the query
    counts for quick tests; robots and scenes are unchanged."""
    rng = np.random.default_rng(1000 + index)
    if index == 1:
        asset = panda_like()
        obbs = random_obbs(rng, 16)
        n = max(1, int(4096 * scale))
        return {"asset": asset, "obbs": obbs, "q": uniform_configs(rng, asset, n),
                "name": "configs_panda7_obb16_n4096"}
    if index == 2:
        asset = panda_like()
        obbs = random_obbs(rng, 64)
        n = max(2, int(65536 * scale))
        frm, to, G = edge_batch(rng, asset, n)
        return {"asset": asset, "obbs": obbs, "from": frm, "to": to, "G": G,
                "name": "edges_panda7_obb64_e65536_linf0.01"}
    if index == 3:
        asset = panda_like()
        obbs = random_obbs(rng, 64)
        B = max(1, int(256 * scale))
        return {"asset": asset, "obbs": obbs, "q": straight_trajectories(rng, asset, B, 64),
                "w": 20.0, "eps": 0.05, "self_margin": 0.01, "delta_t": 0.1,
                "name": "chomp_panda7_obb64_b256_t64"}
    if index == 4:
        asset = fetch_like()
        obbs = random_obbs(rng, 96)
        n_traj, n_roll, T = 32, max(1, int(128 * scale)), 100
        base = straight_trajectories(rng, asset, n_traj, T, noise=0.0)
        L = stomp_noise_L(T, 0.1)
        z = rng.normal(size=(n_traj, n_roll, asset["n_dof"], T))
        noise = np.einsum("ts,brds->brdt", L, z)
        roll = base.transpose(0, 2, 1)[:, None, :, :] + noise   # [traj, roll, D, T]
        lo = np.asarray(asset["joint_lower"])[None, None, :, None]
        hi = np.asarray(asset["joint_upper"])[None, None, :, None]
        roll = np.clip(roll, lo, hi).astype(np.float32).reshape(n_traj * n_roll, asset["n_dof"], T)
        return {"asset": asset, "obbs": obbs, "rollouts": roll, "w": 20.0, "eps": 0.05,
                "self_margin": 0.01, "name": "stomp_fetch8_obb96_32x128x100"}
    if index == 5:
        asset = baxter_like()
        # 128 boxes in a wider, sparser field than workloads 1-4 (centres
        # U([-1.5,1.5]^3), half-extents U(0.02,0.1)): with 110 spheres on two
        # arms the denser field leaves no collision-free edge at all.
        obbs = random_obbs(rng, 128, -1.5, 1.5, 0.02, 0.1)
        esdf = random_esdf(rng)
        n_e = max(2, int(8192 * scale))
        frm, to, G = edge_batch(rng, asset, n_e)
        Ts = rng.integers(32, 129, max(1, int(64 * scale)))
        trajs = [straight_trajectories(rng, asset, 1, int(t))[0] for t in Ts]
        # edge requests of uneven size (16..256 edges), as many planners' batches
        splits = []
        left = n_e
        while left > 0:
            k = min(left, int(rng.integers(16, 257)))
            splits.append(k)
            left -= k
        return {"asset": asset, "obbs": obbs, "esdf": esdf, "from": frm, "to": to, "G": G,
                "edge_splits": splits, "trajectories": trajs, "w": 20.0, "eps": 0.05,
                "self_margin": 0.01, "name": "mixed_baxter14_obb128_esdf128"}
    raise ValueError(f"unknown workload {index}")
