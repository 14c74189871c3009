"""CPU: the oracle and the host-side restatements against the reference's own
outputs (golden vectors made by tests/golden/make_golden.py from the
reference's Python: robot_model_loader.py, planning_scene.py and the FP64
NumPy FK/collision oracle of tests/test_tree_fk_vs_cpu.py)."""
import numpy as np
import pytest

import oracle
from conftest import golden_asset
from prismplan_b200 import _lib, workloads
from prismplan_b200.robot import RobotModelBuilder, build_approx_self_cc_ranges, build_approx_spheres
from prismplan_b200.scene import pack_obbs

ASSETS = ("panda", "fetch", "baxter")


@pytest.mark.parametrize("name", ASSETS)
def test_approx_model_matches_reference_loader(golden, name):
    asset, raw = golden_asset(golden, name)
    a_flat, a_j = build_approx_spheres(asset["spheres_flat"], asset["sphere_to_joint"], asset["n_joints"])
    np.testing.assert_array_equal(np.asarray(a_flat), raw["approx_spheres_flat"])
    np.testing.assert_array_equal(np.asarray(a_j), raw["approx_sphere_to_joint"])
    r = build_approx_self_cc_ranges(asset["self_cc_ranges_flat"], asset["sphere_to_joint"], a_j)
    np.testing.assert_array_equal(np.asarray(r), raw["approx_self_cc_ranges_flat"])


@pytest.mark.parametrize("name", ASSETS)
def test_oracle_fk_matches_reference_numpy(golden, name):
    asset, raw = golden_asset(golden, name)
    om = oracle.OracleModel(RobotModelBuilder.from_asset(asset), np.zeros((0, 4)), np.zeros((0, 8)))
    pos = om.fk_spheres(raw["q"], prec=64)
    ref = raw["fk"][:, :, :3]
    assert np.abs(pos - ref).max() < 1e-12


@pytest.mark.parametrize("name", ASSETS)
def test_inverse_pose_matches_reference(golden, name):
    _, raw = golden_asset(golden, name)
    for s in range(raw["obb_dims"].shape[0]):
        d, p, en = pack_obbs(raw["obb_dims"][s], raw["obb_pos"][s], raw["obb_quat"][s])
        np.testing.assert_allclose(p[:, :3], raw["obb_inv_t"][s], atol=2e-7)
        np.testing.assert_allclose(p[:, 3:7], raw["obb_inv_q"][s], atol=1e-7)
        np.testing.assert_array_equal(d[:, :3], raw["obb_dims"][s].astype(np.float32))


@pytest.mark.parametrize("name", ASSETS)
@pytest.mark.parametrize("gate", [True, False])
def test_oracle_verdicts_match_reference_numpy(golden, name, gate):
    """FP64 two-phase (and ungated) verdicts equal the reference NumPy oracle
    on every (scene, configuration); the only allowed difference is the
    reference oracle's `<=` boundary, which a seeded input never hits."""
    asset, raw = golden_asset(golden, name)
    b = RobotModelBuilder.from_asset(asset)
    flags = 0 if gate else _lib.PS_NO_GATE
    for s in range(raw["obb_dims"].shape[0]):
        d, p, en = pack_obbs(raw["obb_dims"][s], raw["obb_pos"][s], raw["obb_quat"][s])
        om = oracle.OracleModel(b, d, p, en)
        hit, _, gap = om.check_configs(raw["q"], flags=flags, prec=64)
        ref = raw["in_collision"][s]
        bad = np.nonzero(hit.astype(bool) != ref)[0]
        assert len(bad) == 0 or np.abs(gap[bad]).max() < 1e-6, (s, bad, gap[bad])


def test_oracle_masks_follow_reference_rules(golden):
    """Allowed-collision masks in the oracle, by the reference's rules
    (scene_collision.cuh:118-135 skips a box whose mask entry is 0 for the
    sphere's index; :584-606 gives the approximate pass sphere index -1, so it
    applies no mask): all-ones masks change nothing, an all-zero exact mask
    frees every configuration of a box-only scene, and the approximate mask
    changes nothing whatever it holds."""
    asset, raw = golden_asset(golden, "panda")
    b = RobotModelBuilder.from_asset(asset)
    d, p, en = pack_obbs(raw["obb_dims"][0], raw["obb_pos"][0], raw["obb_quat"][0])
    ns, na, no = len(b.sphere_to_joint), len(np.asarray(asset["approx_spheres_flat"])) // 4, len(d)
    om = oracle.OracleModel(b, d, p, en)
    base, _, _ = om.check_configs(raw["q"], prec=64)
    assert 0 < base.sum() < len(base)
    om.set_masks(None, np.ones((ns, no), np.uint8), np.ones((na, no), np.uint8))
    np.testing.assert_array_equal(om.check_configs(raw["q"], prec=64)[0], base)
    om.set_masks(None, None, np.zeros((na, no), np.uint8))
    np.testing.assert_array_equal(om.check_configs(raw["q"], prec=64)[0], base)
    om.set_masks(None, np.zeros((ns, no), np.uint8), None)
    assert om.check_configs(raw["q"], prec=64)[0].sum() == 0


def test_oracle_fp32_baseline_agrees_with_fp64():
    wl = workloads.workload(1, scale=0.25)
    b = RobotModelBuilder.from_asset(wl["asset"])
    om = oracle.OracleModel(b, *wl["obbs"])
    h64, c64, gap = om.check_configs(wl["q"], flags=_lib.PS_CLEARANCE_OBB, prec=64)
    h32, c32, _ = om.check_configs(wl["q"], flags=_lib.PS_CLEARANCE_OBB, prec=32, want_gap=False)
    flips = np.nonzero(h64 != h32)[0]
    assert len(flips) == 0 or np.abs(gap[flips]).max() < 1e-5
    assert np.abs(c64 - c32).max() < 1e-5


def test_control_cost_matrix():
    for T in (8, 51, 64, 100):
        R = oracle.control_cost_R(T, 0.1)
        np.testing.assert_allclose(R, workloads.control_cost_R(T, 0.1), rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(R, R.T, atol=1e-9)
        # 9-band: the 5-point acceleration stencil squared
        i, j = np.nonzero(np.abs(R) > 0)
        assert np.abs(i - j).max() <= 4


def test_edge_oracle_samples_are_configs():
    """An edge is invalid iff one of its samples t=j/G (FP32 product-sum) is,
    or, when G % 16 != 0, its start configuration (edge_eval.cuh:110-130)."""
    wl = workloads.workload(2, scale=0.002)
    b = RobotModelBuilder.from_asset(wl["asset"])
    om = oracle.OracleModel(b, *wl["obbs"])
    frm, to, G = wl["from"][:24], wl["to"][:24], np.minimum(wl["G"][:24], 64)
    valid, cost, _, _, _ = om.check_edges(frm, to, G, early_exit=False)
    for e in range(len(frm)):
        t = (np.arange(1, G[e] + 1, dtype=np.float32) / np.float32(G[e])).astype(np.float32)
        if G[e] % 16:   # the reference's padding slots evaluate the start configuration
            t = np.append(t, np.float32(0.0))
        q = (frm[e][None] + t[:, None] * (to[e] - frm[e])[None]).astype(np.float32)
        hit, _, _ = om.check_configs(q, prec=64, want_gap=False)
        assert bool(valid[e]) == (not hit.any())
        if valid[e]:
            assert abs(cost[e] - np.linalg.norm((to[e] - frm[e]).astype(np.float64))) < 1e-5


def test_workload_shapes():
    w1 = workloads.workload(1)
    assert w1["q"].shape == (4096, 7) and w1["obbs"][0].shape == (16, 4)
    assert len(w1["asset"]["sphere_to_joint"]) == 59
    w2 = workloads.workload(2)
    assert w2["from"].shape == (65536, 7) and w2["G"].min() >= 1 and w2["G"].max() <= 600
    assert w2["obbs"][0].shape == (64, 4)
    w3 = workloads.workload(3)
    assert w3["q"].shape == (256, 64, 7)
    w4 = workloads.workload(4, scale=0.05)
    assert w4["rollouts"].shape[1:] == (8, 100) and len(w4["asset"]["sphere_to_joint"]) == 70
    a5 = workloads.baxter_like()
    assert a5["n_dof"] == 14 and len(a5["sphere_to_joint"]) == 110 and a5["joint_parents"][8] == 0
