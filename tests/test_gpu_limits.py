"""Size limits at their maximum, against the reference kernels run on the
same inputs, and one past each refused with PS_EINVAL:

* PS_MAX_OBBS = 1024 boxes: config verdicts and OBB clearance, edges
  (persistent and plain), waypoint costs;
* PS_MAX_LAYERS = 8 ESDF layers: config verdicts and ESDF clearance, edges;
* PS_MAX_DOF = 14: a 14-DoF chain with 112 spheres (generic rotations, one
  prismatic joint): FK, config verdicts, edges, waypoint costs;
* the self check's shared-memory bound: a model too large for it is refused
  with the sizes in the message, and the same model without the self check
  still runs.
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import golden_asset
from prismplan_b200 import _lib, api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu

COST = dict(w=2.0, wm=0.05, sm=0.01)


def _cost_params():
    return api.CostParams(collision_cost_weight=COST["w"], world_collision_margin=COST["wm"],
                          self_collision_margin=COST["sm"])


@pytest.fixture(scope="module")
def panda(golden):
    asset, _ = golden_asset(golden, "panda")
    return asset, RobotModelBuilder.from_asset(asset).build()


def _configs_match(b, sc, ref, q, clearance=None):
    hit, clr = api.check_configs(b, sc, torch.from_numpy(q).cuda(), clearance=clearance)
    rhit, _ = ref.check_configs(q)
    np.testing.assert_array_equal(hit.cpu().numpy(), rhit)
    return rhit, clr


def _edges_match(b, sc, ref, frm, to, G):
    rv, rc, _ = ref.check_edges(frm, to, G)
    for persistent in (True, False):
        v, c, _ = api.check_edges(b, sc, frm, to, samples=G, persistent=persistent)
        np.testing.assert_array_equal(v.cpu().numpy(), rv, err_msg=f"persistent={persistent}")
        assert np.array_equal(c.cpu().numpy().view(np.uint32), rc.view(np.uint32))
    return rv


def _costs_match(b, sc, ref, th):
    wp, _, _ = api.traj_cost(b, sc, torch.from_numpy(th).cuda(), _cost_params(), want_grad=False)
    rsc, _, _ = ref.chomp(th.transpose(0, 2, 1), COST["w"], COST["wm"], COST["sm"], grad=False)
    ours, theirs = wp.cpu().numpy().reshape(-1), rsc[:, 0, :].reshape(-1)
    rel = np.abs(ours - theirs) / np.maximum(np.abs(theirs), 1.0)
    assert rel.max() < 1e-3, rel.max()
    return rel.max(), (theirs > 0).mean()


def test_max_boxes(panda):
    asset, b = panda
    rng = np.random.default_rng(1024)
    obbs = workloads.random_obbs(rng, _lib.PS_MAX_OBBS, lo=-1.5, hi=1.5, half_lo=0.005, half_hi=0.03)
    sc = SceneTensors(*obbs)
    ref = oracle.RefKernels(b, *obbs)
    q = workloads.uniform_configs(np.random.default_rng(1), asset, 512)
    rhit, clr = _configs_match(b, sc, ref, q, clearance="obb")
    assert 0.05 < rhit.mean() < 0.95
    err = np.abs(clr.cpu().numpy() - ref.obb_min_clearance(q)).max()
    assert err < 1e-5
    frm, to, G = workloads.edge_batch(np.random.default_rng(2), asset, 128, step=0.02, max_samples=64)
    rv = _edges_match(b, sc, ref, frm, to, G)
    rel, active = _costs_match(b, sc, ref, workloads.straight_trajectories(rng, asset, 8, 16))
    print(f"{_lib.PS_MAX_OBBS} boxes: hit {rhit.mean():.2f}, OBB clearance err {err:.1e} m, edges valid "
          f"{rv.mean():.2f}, cost rel diff {rel:.1e} (active {active:.2f})")
    over = SceneTensors(*workloads.random_obbs(rng, _lib.PS_MAX_OBBS + 1))
    with pytest.raises(_lib.PrismError):
        api.check_configs(b, over, torch.from_numpy(q[:4]).cuda())


def test_max_layers(panda):
    asset, b = panda
    rng = np.random.default_rng(8)
    centres = [(0.55 * np.cos(a), 0.55 * np.sin(a), 0.45)
               for a in np.linspace(0.0, 2.0 * np.pi, _lib.PS_MAX_LAYERS, endpoint=False)]
    layers = [workloads.random_esdf(rng, n_vox=24, voxel=0.04, n_boxes=3, centre=c) for c in centres]
    esdf = tuple(np.concatenate(x) for x in zip(*layers))
    obbs = workloads.random_obbs(rng, 8)
    sc = SceneTensors(*obbs, *esdf)
    ref = oracle.RefKernels(b, *obbs, esdf=esdf)
    q = workloads.uniform_configs(np.random.default_rng(1), asset, 512)
    rhit, clr = _configs_match(b, sc, ref, q, clearance="esdf")
    assert 0.05 < rhit.mean() < 0.95
    err = np.abs(clr.cpu().numpy() - ref.esdf_min_clearance(q)).max()
    assert err < 1e-5
    frm, to, G = workloads.edge_batch(np.random.default_rng(2), asset, 128, step=0.02, max_samples=64)
    rv = _edges_match(b, sc, ref, frm, to, G)
    print(f"{_lib.PS_MAX_LAYERS} ESDF layers: hit {rhit.mean():.2f}, ESDF clearance err {err:.1e} m, "
          f"edges valid {rv.mean():.2f}")
    extra = workloads.random_esdf(rng, n_vox=24, voxel=0.04, n_boxes=3)
    nine = tuple(np.concatenate([x, y]) for x, y in zip(esdf, extra))
    with pytest.raises(_lib.PrismError):
        api.check_configs(b, SceneTensors(*obbs, *nine), torch.from_numpy(q[:4]).cuda())


def test_max_dof_chain():
    asset = workloads.generic_chain(seed=1014, n_links=_lib.PS_MAX_DOF, spheres_per_link=8)
    b = RobotModelBuilder.from_asset(asset).build()
    obbs = workloads.random_obbs(np.random.default_rng(14), 24, lo=-1.2, hi=1.2, half_lo=0.02, half_hi=0.06)
    sc = SceneTensors(*obbs)
    ref = oracle.RefKernels(b, *obbs)
    q = workloads.uniform_configs(np.random.default_rng(3), asset, 512)
    ours = api.fk_spheres(b, torch.from_numpy(q).cuda()).cpu().numpy()
    assert np.array_equal(ours.view(np.uint32), ref.fk_spheres(q).view(np.uint32))
    rhit, _ = _configs_match(b, sc, ref, q)
    assert 0.05 < rhit.mean() < 0.95
    frm, to, G = workloads.edge_batch(np.random.default_rng(4), asset, 128, step=0.02, max_samples=48)
    rv = _edges_match(b, sc, ref, frm, to, G)
    rel, active = _costs_match(b, sc, ref, workloads.straight_trajectories(np.random.default_rng(5), asset, 8, 16))
    print(f"{_lib.PS_MAX_DOF}-DoF chain, {len(b.sphere_to_joint)} spheres: hit {rhit.mean():.2f}, edges valid "
          f"{rv.mean():.2f}, cost rel diff {rel:.1e} (active {active:.2f})")
    with pytest.raises(_lib.PrismError):
        RobotModelBuilder.from_asset(workloads.generic_chain(seed=1014, n_links=_lib.PS_MAX_DOF + 1)).build()


def test_self_check_size_bound():
    """A 14-link chain with 24 spheres per link (336 spheres) is past the
    self check's shared-memory bound: the self check is refused with the
    sizes in the message; without it the same model runs."""
    asset = workloads.generic_chain(seed=1015, n_links=_lib.PS_MAX_DOF, spheres_per_link=24)
    b = RobotModelBuilder.from_asset(asset).build()
    q = torch.from_numpy(workloads.uniform_configs(np.random.default_rng(6), asset, 64)).cuda()
    with pytest.raises(_lib.PrismError, match="check_self"):
        api.check_configs(b, None, q, check_self=True)
    with pytest.raises(_lib.PrismError, match="check_self"):
        api.check_edges(b, None, q[:32], q[32:], samples=np.full(32, 8, np.int32),
                        params=api.EdgeEvalParams(check_self=True))
    hit, _ = api.check_configs(b, None, q)
    assert int(hit.sum()) == 0
