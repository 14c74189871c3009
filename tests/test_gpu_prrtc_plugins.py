"""GPU: the planner plugins' substrate calls, in the reference's own call
shapes, on its MotionBenchMaker sample, bit-exact against the reference
kernels.

tests/golden/mbm_sample_fixtures.npz (made by tests/golden/make_mbm_fixtures.py
from the reference's code) holds what the plugins hand the substrate: the
prrtc.RobotModelBuilder fields that build_robot_model sets for the Panda
(robot_model_loader.py:193-243) and, per sample problem, the
prrtc.SceneCollisionDataBuilder fields and the OBB arrays behind them that
PlanningScene.build_scene_collision_data fills (planning_scene.py:189-242),
with the problem's start and goal. Here the same fields are set on
prismplan_b200.prrtc's builders, and the calls are made with the keywords of
_SubstratePlannerBase._preflight (_substrate_planner_base.py:281-292) and
through EdgeEvalGpu (edge_batch_bridge.hh:60-96).
"""
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
from prismplan_b200 import api, prrtc, workloads

pytestmark = pytest.mark.gpu

FIX = Path(__file__).resolve().parent / "golden" / "mbm_sample_fixtures.npz"


def _robot(z):
    r = prrtc.RobotModelBuilder()
    for k in z["robot_fields"].tolist():
        v = z[f"robot/{k}"]
        setattr(r, k, v.item() if v.ndim == 0 else v.tolist())   # pybind std::vector / int fields
    return r.build()


def _scene(z, n):
    dims = torch.from_numpy(z[f"p{n}/obb_dims"]).cuda().contiguous()
    pose = torch.from_numpy(z[f"p{n}/obb_pose"]).cuda().contiguous()
    en = torch.from_numpy(z[f"p{n}/obb_enable"]).cuda().contiguous()
    sb = prrtc.SceneCollisionDataBuilder()
    ptrs = {"obb_dims_ptr": dims.data_ptr(), "obb_pose_ptr": pose.data_ptr(), "obb_enable_ptr": en.data_ptr(),
            "n_obbs": int(z[f"p{n}/n_obbs"])}
    for k in z[f"p{n}/scene_fields"].tolist():   # exactly the fields the reference's scene sets
        setattr(sb, k, ptrs[k])
    return sb, (dims, pose, en)


@pytest.fixture(scope="module")
def fixtures():
    z = np.load(FIX)
    return z, _robot(z)


def _asset_limits(robot):
    return np.asarray(robot.joint_lower, np.float32), np.asarray(robot.joint_upper, np.float32)


@pytest.mark.parametrize("n", [0, 1, 2])
def test_preflight_call_shape_bitexact(fixtures, n):
    z, robot = fixtures
    sb, keep = _scene(z, n)
    lo, hi = _asset_limits(robot)
    rng = np.random.default_rng(300 + n)
    start, goal = z[f"p{n}/start"], z[f"p{n}/goal"]
    configs = np.concatenate([start[None], goal[None],
                              rng.uniform(lo, hi, (4094, len(lo))).astype(np.float32)])
    hits = prrtc.check_collision_scene(configs=np.asarray(configs, dtype=np.float32), scene=sb, robot=robot,
                                       collision_margin=0.0)
    assert hits.dtype == bool and hits.shape == (len(configs),)
    ref = oracle.RefKernels(robot, z[f"p{n}/obb_dims"], z[f"p{n}/obb_pose"], z[f"p{n}/obb_enable"])
    rhit, _ = ref.check_configs(configs)
    np.testing.assert_array_equal(hits, rhit.astype(bool))
    assert not hits[0] and not hits[1], "the sample's start and goal are collision-free"
    print(f"problem {n} ({z[f'p{n}/scene_name']}): {hits[2:].mean():.3f} of random configurations collide")
    assert 0.0 < hits[2:].mean() < 1.0
    del keep


@pytest.mark.parametrize("n", [0, 1, 2])
def test_edge_bridge_bitexact(fixtures, n):
    z, robot = fixtures
    sb, keep = _scene(z, n)
    lo, hi = _asset_limits(robot)
    rng = np.random.default_rng(400 + n)
    D = len(lo)
    start, goal = z[f"p{n}/start"], z[f"p{n}/goal"]
    # the straight start -> goal edge, and edges between points along it with noise
    a = rng.uniform(0.0, 1.0, (2047, 1)).astype(np.float32)
    b = np.clip(a + rng.uniform(-0.3, 0.3, a.shape).astype(np.float32), 0.0, 1.0)
    noise = lambda: rng.normal(0.0, 0.3, (len(a), D)).astype(np.float32)  # noqa: E731
    frm = np.clip(start + a * (goal - start) + noise(), lo, hi).astype(np.float32)
    to = np.clip(start + b * (goal - start) + noise(), lo, hi).astype(np.float32)
    frm = np.concatenate([start[None], frm])
    to = np.concatenate([goal[None], to])
    G = workloads.linf_samples(frm, to, 0.01)
    ev = api.EdgeEvalGpu(D, len(frm), sb, robot)
    params = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    valid, cost, _ = ev.evaluate(frm.reshape(-1), to.reshape(-1), len(frm), params)
    ref = oracle.RefKernels(robot, z[f"p{n}/obb_dims"], z[f"p{n}/obb_pose"], z[f"p{n}/obb_enable"])
    rv, rc, _ = ref.check_edges(frm, to, G)
    np.testing.assert_array_equal(valid, rv)
    assert np.array_equal(cost.view(np.uint32), rc.view(np.uint32))
    print(f"problem {n}: straight start->goal edge valid={bool(valid[0])}; {valid.mean():.3f} of edges valid")
    assert 0.0 < valid.mean() < 1.0
    del keep
