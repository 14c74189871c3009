"""Generate tests/golden/reference_golden.npz from the reference's own Python.

Run in a container that has the read-only reference checkout:

    python tests/golden/make_golden.py <reference root>
    (or PRISMPLAN_REF=<reference root> python tests/golden/make_golden.py)

It imports, from the reference (paths inside code/gpu_planning/):
  * python/gpu_planning/substrate/robot_model_loader.py  -- load_robot_asset
    (YAML parse + approximate-sphere / approximate self-range derivation)
  * python/gpu_planning/substrate/planning_scene.py      -- _inverse_pose
  * tests/test_tree_fk_vs_cpu.py                          -- fk_spheres (FP64
    tree FK) and in_collision (FP64 sphere-vs-OBB), the reference's own CPU
    oracle for this path
and records their outputs on seeded inputs for the three shipped robot assets
(panda, fetch, baxter). The GPU box has no reference checkout: tests read only
the committed .npz.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "reference_golden.npz"


def _import_file(name: str, path: Path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(ref_root: str) -> None:
    gp = Path(ref_root) / "code" / "gpu_planning"
    sys.path.insert(0, str(gp / "python"))
    from gpu_planning.substrate import planning_scene as ps_mod  # noqa: E402
    from gpu_planning.substrate import robot_model_loader as loader  # noqa: E402

    fkmod = _import_file("ref_tree_fk_vs_cpu", gp / "tests" / "test_tree_fk_vs_cpu.py")
    rng = np.random.default_rng(20261203)
    out = {}
    for name in ("panda", "fetch", "baxter"):
        asset = loader.load_robot_asset(str(gp / "config" / "robots" / f"{name}.yaml"))
        for k in ("fixed_transforms", "joint_types", "spheres_flat", "sphere_to_joint",
                  "self_cc_ranges_flat", "joint_lower", "joint_upper", "joint_parents",
                  "joint_id_to_dof", "t_memory_idx", "dfs_order", "approx_spheres_flat",
                  "approx_sphere_to_joint", "approx_self_cc_ranges_flat"):
            out[f"{name}/{k}"] = np.asarray(asset[k])
        out[f"{name}/n_dof"] = np.asarray(asset["n_dof"])
        out[f"{name}/n_joints"] = np.asarray(asset["n_joints"])
        # The device model holds FP32 constants: evaluate the reference oracle on
        # the FP32-rounded transforms and spheres (values, not formulas, change).
        asset32 = dict(asset)
        for k in ("fixed_transforms", "spheres_flat"):
            asset32[k] = [float(v) for v in np.asarray(asset[k], np.float32)]
        lo = np.asarray(asset["joint_lower"], np.float64)
        hi = np.asarray(asset["joint_upper"], np.float64)
        q = (lo + rng.random((48, len(lo))) * (hi - lo)).astype(np.float32)
        out[f"{name}/q"] = q
        out[f"{name}/fk"] = np.stack([fkmod.fk_spheres(asset32, c.astype(np.float64)) for c in q])
        # six random OBB worlds of 8 boxes around the robot
        scenes_d, scenes_p, scenes_q, verdicts, inv_t, inv_q = [], [], [], [], [], []
        for _ in range(6):
            dims = rng.uniform(0.04, 0.3, (8, 3))
            pos = rng.uniform(-1.0, 1.0, (8, 3)) + np.array([0.0, 0.0, 0.4])
            qq = rng.normal(size=(8, 4))
            qq /= np.linalg.norm(qq, axis=1, keepdims=True)
            obbs = [(dims[i], pos[i], qq[i]) for i in range(8)]
            obbs32 = [(d.astype(np.float32).astype(np.float64), pp, qv) for d, pp, qv in obbs]
            verdicts.append([fkmod.in_collision(fkmod.fk_spheres(asset32, c.astype(np.float64)), obbs32) for c in q])
            ts, qs = zip(*[ps_mod._inverse_pose(pos[i], qq[i]) for i in range(8)])
            scenes_d.append(dims)
            scenes_p.append(pos)
            scenes_q.append(qq)
            inv_t.append(np.stack(ts))
            inv_q.append(np.stack(qs))
        out[f"{name}/obb_dims"] = np.stack(scenes_d)
        out[f"{name}/obb_pos"] = np.stack(scenes_p)
        out[f"{name}/obb_quat"] = np.stack(scenes_q)
        out[f"{name}/obb_inv_t"] = np.stack(inv_t)
        out[f"{name}/obb_inv_q"] = np.stack(inv_q)
        out[f"{name}/in_collision"] = np.asarray(verdicts, bool)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    import os

    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PRISMPLAN_REF")
    if not root:
        sys.exit("usage: make_golden.py <reference root> (or set PRISMPLAN_REF)")
    main(root)
