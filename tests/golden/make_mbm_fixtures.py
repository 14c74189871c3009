"""Generate tests/golden/mbm_sample_fixtures.npz: the substrate call shapes of
the reference's planner plugins on its 3-problem MotionBenchMaker sample.

Run in a container that has the read-only reference checkout:

    python tests/golden/make_mbm_fixtures.py <reference root>
    (or PRISMPLAN_REF=<reference root> python tests/golden/make_mbm_fixtures.py)

The plugins reach the substrate through three prrtc names
(code/gpu_planning/python/gpu_planning/plugins/_substrate_planner_base.py:
build_robot_model at :219, PlanningScene.build_scene_collision_data at :266,
prrtc.check_collision_scene in _preflight at :281-292). This script runs the
reference's own code for the first two on the sample problems:

  * benchmark/loaders.py:76       load_vamp_problems (examples/data/
                                  sample_mbm_problems.json)
  * benchmark/problem.py:122      obstacle_to_obb, obstacles_to_obbs
  * substrate/planning_scene.py   PlanningScene.update_world, _rebuild_tensors,
                                  build_scene_collision_data (device "cpu")
  * substrate/robot_model_loader.py:193  build_robot_model (config/robots/panda.yaml)

with a recording stand-in registered as the `prrtc` module, so that every
attribute those functions set on prrtc.RobotModelBuilder and
prrtc.SceneCollisionDataBuilder is captured, together with the host arrays
behind the scene's device pointers. The GPU box has no reference checkout:
tests read only the committed .npz.
"""
from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "mbm_sample_fixtures.npz"


class _Recorder:
    """Records every attribute set on it; build()/destroy() do nothing."""

    def __init__(self):
        object.__setattr__(self, "fields", {})

    def __setattr__(self, k, v):
        self.fields[k] = v

    def __getattr__(self, k):
        if k in ("build", "build_on_device", "destroy", "update_joint_limits"):
            return lambda *a, **kw: self
        if k in self.fields:
            return self.fields[k]
        if k in ("joint_parents", "joint_id_to_dof", "t_memory_idx", "dfs_order"):
            return []   # the tree fields exist, as on the current prrtc
        raise AttributeError(k)


def main(ref_root: str) -> None:
    gp = Path(ref_root) / "code" / "gpu_planning"
    sys.path.insert(0, str(gp / "python"))
    stub = types.ModuleType("prrtc")
    stub.RobotModelBuilder = _Recorder
    stub.SceneCollisionDataBuilder = _Recorder
    sys.modules["prrtc"] = stub

    from gpu_planning.benchmark import load_vamp_problems, obstacles_to_obbs  # noqa: E402
    from gpu_planning.substrate.planning_scene import PlanningScene  # noqa: E402
    from gpu_planning.substrate.robot_model_loader import build_robot_model  # noqa: E402

    out = {}
    robot = build_robot_model(str(gp / "config" / "robots" / "panda.yaml"))
    names = sorted(robot.fields)
    out["robot_fields"] = np.asarray(names)
    for k in names:
        out[f"robot/{k}"] = np.asarray(robot.fields[k])

    problems = load_vamp_problems(str(gp / "examples" / "data" / "sample_mbm_problems.json"))
    out["n_problems"] = np.asarray(len(problems))
    for n, prob in enumerate(problems):
        scene = PlanningScene(num_joints=len(prob.start), device="cpu")
        scene.update_world(obstacles_to_obbs(prob.obstacles))
        with scene._voxel_plan_lock:
            builder = scene.build_scene_collision_data()
        out[f"p{n}/scene_fields"] = np.asarray(sorted(builder.fields))
        out[f"p{n}/n_obbs"] = np.asarray(builder.fields["n_obbs"])
        # the host arrays behind the device pointers the builder was given
        out[f"p{n}/obb_dims"] = scene._obb_dims_t.numpy().copy()
        out[f"p{n}/obb_pose"] = scene._obb_pose_t.numpy().copy()
        out[f"p{n}/obb_enable"] = scene._obb_enable_t.numpy().copy()
        out[f"p{n}/start"] = np.asarray(prob.start, np.float32)
        out[f"p{n}/goal"] = np.asarray(prob.goal, np.float32)
        out[f"p{n}/scene_name"] = np.asarray(prob.scene)
        print(f"problem {n}: scene {prob.scene}, {builder.fields['n_obbs']} OBBs, "
              f"builder fields {sorted(builder.fields)}")
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({len(problems)} problems, robot fields {names})")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PRISMPLAN_REF")
    if not root:
        sys.exit("usage: make_mbm_fixtures.py <reference root> (or set PRISMPLAN_REF)")
    main(root)
