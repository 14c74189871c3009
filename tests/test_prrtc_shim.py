"""The substrate names of the reference's `prrtc` module (bindings.cpp:960-1037,
used by python/gpu_planning/plugins/_substrate_planner_base.py:281-292) exist
in prismplan_b200.prrtc with the same fields and keywords. CPU only."""
import inspect

import pytest

from prismplan_b200 import prrtc

ROBOT_FIELDS = (
    "n_dof n_joints fixed_transforms joint_types spheres_flat sphere_to_joint self_cc_ranges_flat "
    "approx_spheres_flat approx_sphere_to_joint approx_self_cc_ranges_flat approx_fixed_transforms "
    "approx_joint_types joint_lower joint_upper joint_parents joint_id_to_dof t_memory_idx dfs_order "
    "mesh_bvh_nodes mesh_tri_vertices mesh_link_bvh_root mesh_link_tri_offset mesh_link_tri_count").split()
SCENE_FIELDS = (
    "obb_dims_ptr obb_pose_ptr obb_enable_ptr n_obbs voxel_params_ptr voxel_pose_ptr voxel_enable_ptr "
    "voxel_features_ptr n_voxel_layers max_voxels_per_layer sphere_acm_mask_ptr sphere_obb_acm_mask_ptr "
    "sphere_obb_acm_mask_approx_ptr").split()


def test_robot_builder_fields_and_methods():
    r = prrtc.RobotModelBuilder()
    for f in ROBOT_FIELDS:
        assert hasattr(r, f), f
        setattr(r, f, getattr(r, f))   # writable, like def_readwrite
    for m in ("build", "update_joint_limits", "destroy"):
        assert callable(getattr(r, m)), m


def test_scene_builder_fields():
    s = prrtc.SceneCollisionDataBuilder()
    for f in SCENE_FIELDS:
        assert hasattr(s, f), f
        setattr(s, f, getattr(s, f))


def test_check_collision_scene_keywords():
    # the plugins call it with configs=, scene=, robot=, collision_margin=
    params = inspect.signature(prrtc.check_collision_scene).parameters
    assert list(params)[:4] == ["configs", "scene", "robot", "collision_margin"]
    assert params["collision_margin"].default == 0.0


def test_planner_entry_points_are_refused():
    for name in ("solve_scene", "chomp_solve_scene", "stomp_solve_scene", "CHOMPSettings"):
        with pytest.raises(AttributeError, match="substrate"):
            getattr(prrtc, name)


def test_planning_scene_surface(tmp_path):
    # the members the planner plugins read (planning_scene.py:92-128), host side only
    from prismplan_b200.scene import PlanningScene

    yaml_text = "\n".join([
        "name: two_link", "n_dof: 2", "n_joints: 3",
        "joint_types: [-1, 5, 5]",
        "fixed_transforms:",
        "  - [1,0,0,0, 0,1,0,0, 0,0,1,0, 0,0,0,1]",
        "  - [1,0,0,0, 0,1,0,0, 0,0,1,0.1, 0,0,0,1]",
        "  - [1,0,0,0.3, 0,1,0,0, 0,0,1,0, 0,0,0,1]",
        "spheres: [[0,0,0,0.05], [0.1,0,0,0.05], [0.1,0,0,0.04]]",
        "sphere_to_joint: [1, 1, 2]",
        "self_cc_ranges: []",
        "joint_lower: [-1, -1]", "joint_upper: [1, 1]",
    ])
    path = tmp_path / "two_link.yaml"
    path.write_text(yaml_text)
    scene = PlanningScene.from_robot_asset(str(path), device="cpu")
    assert scene.num_joints == 2 and scene.robot_id == "two_link" and scene.n_obbs == 0
    scene.add_cuboid("a", [0.1, 0.2, 0.3], [1.0, 0.0, 0.5])
    scene.add_cuboid("b", [0.2, 0.2, 0.2], [0.0, 1.0, 0.5], [0.0, 1.0, 0.0, 0.0])
    obs = scene.current_obstacles
    assert [o["name"] for o in obs] == ["a", "b"] and obs[1]["quaternion"] == [0.0, 1.0, 0.0, 0.0]
    assert obs[0]["type"] == "cuboid" and obs[0]["dims"] == [0.1, 0.2, 0.3]
    clone = PlanningScene(2)
    clone.update_world(obs)
    assert clone.current_obstacles == obs


def test_scene_tensors_masks_host_side():
    """Allowed-collision masks on SceneTensors (host side, CPU tensors): rows
    of the right width are kept and pointed at, a ragged mask is refused, and
    `masks` hands them to the oracle under its names."""
    import numpy as np

    from prismplan_b200 import workloads
    from prismplan_b200.scene import SceneTensors

    rng = np.random.default_rng(3)
    obbs = workloads.random_obbs(rng, 5)
    m_obb = (rng.random((7, 5)) > 0.5).astype(np.uint8)
    m_apx = np.zeros((3, 5), np.uint8)
    sc = SceneTensors(*obbs, device="cpu", sphere_obb_acm_mask=m_obb, sphere_obb_acm_mask_approx=m_apx.ravel())
    v = sc.view()
    assert v.sphere_obb_acm_mask and v.sphere_obb_acm_mask_approx and not v.sphere_acm_mask
    np.testing.assert_array_equal(sc.tensors["sphere_obb_acm_mask"].numpy(), m_obb)
    assert set(sc.masks) == {"obb_acm", "obb_acm_apx"} and sc.masks["obb_acm_apx"].shape == (3, 5)
    with pytest.raises(ValueError):
        SceneTensors(*obbs, device="cpu", sphere_obb_acm_mask=np.ones(11, np.uint8))
    with pytest.raises(ValueError):   # no ESDF layers: an ESDF mask has no columns
        SceneTensors(*obbs, device="cpu", sphere_acm_mask=np.ones(4, np.uint8))


def test_reference_call_shapes_set_only_known_fields():
    """Every field the reference's build_robot_model and
    PlanningScene.build_scene_collision_data set on the prrtc builders
    (recorded in tests/golden/mbm_sample_fixtures.npz) exists on this
    module's builders."""
    from pathlib import Path

    import numpy as np

    z = np.load(Path(__file__).resolve().parent / "golden" / "mbm_sample_fixtures.npz")
    robot_fields = z["robot_fields"].tolist()
    assert set(robot_fields) <= set(ROBOT_FIELDS)
    assert {"n_dof", "fixed_transforms", "spheres_flat", "joint_parents"} <= set(robot_fields)
    for n in range(int(z["n_problems"])):
        fields = z[f"p{n}/scene_fields"].tolist()
        assert set(fields) <= set(SCENE_FIELDS), fields
        assert int(z[f"p{n}/n_obbs"]) == len(z[f"p{n}/obb_dims"]) > 0
