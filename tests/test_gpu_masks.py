"""Allowed-collision masks (scene_collision_data.hh: sphere_acm_mask,
sphere_obb_acm_mask, sphere_obb_acm_mask_approx; 0 = pair ignored) through
every path that reads them, against PrismPlan's own kernels run on the same
scene and masks: config verdicts, OBB and ESDF clearance, edge verdicts and
costs (persistent, plain, mixed batch), the edge ESDF clearance, waypoint and
rollout costs, and the cost gradient against FP64 finite differences.

The approximate mask is all zeros here: the reference's approximate pass
looks no mask up (scene_collision.cuh:584-606 passes sphere index -1 to
sphere_scene_in_collision), so a gate that applied it would pass every
configuration the scene's boxes collide with."""
import numpy as np
import pytest
from conftest import COST_REL_TOL, assert_gradient_vs_fd
import torch

import oracle
from conftest import golden_asset
from prismplan_b200 import api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu


def three_layer_esdf(rng):
    """Three ESDF layers, the middle one disabled: mask columns follow the
    layers' own indices."""
    a = workloads.random_esdf(rng, n_vox=48, voxel=0.02, centre=(0.45, 0.0, 0.45))
    c = workloads.random_esdf(rng, n_vox=48, voxel=0.02, centre=(0.2, 0.35, 0.6))
    off = workloads.random_esdf(np.random.default_rng(5), n_vox=48, voxel=0.02, centre=(0.2, 0.35, 0.6))
    out = tuple(np.concatenate(x) for x in zip(a, off, c))
    out[2][1] = 0
    return out


@pytest.fixture(scope="module")
def case(golden):
    asset, _ = golden_asset(golden, "panda")
    rng = np.random.default_rng(77)
    obbs = workloads.random_obbs(rng, 16)
    obbs[2][[3, 9]] = 0        # disabled boxes: the masks index the boxes as given
    esdf = three_layer_esdf(rng)
    b = RobotModelBuilder.from_asset(asset).build()
    ns = len(b.sphere_to_joint)
    na = len(np.asarray(asset["approx_spheres_flat"]).reshape(-1, 4))
    masks = {
        "sphere_acm_mask": (rng.random((ns, 3)) > 0.5).astype(np.uint8),
        "sphere_obb_acm_mask": (rng.random((ns, 16)) > 0.5).astype(np.uint8),
        "sphere_obb_acm_mask_approx": np.zeros((na, 16), np.uint8),
    }
    sc = SceneTensors(*obbs, *esdf, **masks)
    ref = oracle.RefKernels(b, *obbs, esdf=esdf, masks=sc.masks)
    ref_open = oracle.RefKernels(b, *obbs, esdf=esdf)
    return asset, obbs, esdf, b, sc, ref, ref_open, masks


def test_config_verdicts_with_masks(case):
    asset, obbs, esdf, b, sc, ref, ref_open, _ = case
    q = workloads.uniform_configs(np.random.default_rng(1), asset, 4096)
    hit, _ = api.check_configs(b, sc, torch.from_numpy(q).cuda())
    rhit, _ = ref.check_configs(q)
    open_hit, _ = ref_open.check_configs(q)
    hit = hit.cpu().numpy()
    print(f"hit rate with masks {rhit.mean():.3f}, without {open_hit.mean():.3f}")
    assert (rhit != open_hit).any() and 0.05 < rhit.mean() < 0.95
    np.testing.assert_array_equal(hit, rhit)


def test_config_obb_clearance_with_masks(case):
    asset, obbs, esdf, b, sc, ref, _, _ = case
    q = workloads.uniform_configs(np.random.default_rng(2), asset, 1024)
    _, clr = api.check_configs(b, sc, torch.from_numpy(q).cuda(), clearance="obb")
    rclr = ref.obb_min_clearance(q)
    err = np.abs(clr.cpu().numpy() - rclr).max()
    print(f"masked OBB clearance: max |ours - reference| = {err:.2e} m")
    assert err < 1e-5


def test_edges_with_masks(case):
    asset, obbs, esdf, b, sc, ref, _, _ = case
    frm, to, G = workloads.edge_batch(np.random.default_rng(3), asset, 1536, step=0.02, max_samples=200)
    G[:4] = [0, 1, 16, 33]
    rv, rc, _ = ref.check_edges(frm, to, G)
    assert 0.05 < rv.mean() < 0.95
    f, t, g = (torch.from_numpy(x).cuda() for x in (frm, to, G))
    for persistent in (True, False):
        v, c, _ = api.check_edges(b, sc, f, t, samples=g, persistent=persistent)
        np.testing.assert_array_equal(v.cpu().numpy(), rv, err_msg=f"persistent={persistent}")
        assert np.array_equal(c.cpu().numpy().view(np.uint32), rc.view(np.uint32))
    batch = api.MixedBatch(b, 2, len(G), 0, 0, 0)
    cut = 700
    outs = [batch.add_edges(f[:cut], t[:cut], g[:cut]), batch.add_edges(f[cut:], t[cut:], g[cut:])]
    batch.launch(sc, api.EdgeEvalParams(), api.CostParams())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(torch.cat([o[0] for o in outs]).cpu().numpy(), rv)
    batch.close()


def test_esdf_clearance_with_masks(case):
    """Config ESDF min-clearance against the reference's
    scene_min_clearance_runtime (run in 4-thread blocks), and the edge
    clearance of every path against the min of the config clearance over the
    edge's samples j = 1..G, formed as the kernels form them (t = j / G,
    q = fma(t, to - from, from)). The reference's own edge clearance
    (evaluate_edges_batch with compute_clearance) is not run: its 64-thread
    blocks call that function's __shfl_xor_sync(0xf, ...) from lanes outside
    the mask (scene_collision.cuh:379), which CUDA leaves undefined."""
    asset, obbs, esdf, b, sc, ref, _, _ = case
    frm, to, G = workloads.edge_batch(np.random.default_rng(4), asset, 384, step=0.02, max_samples=120)
    G[:3] = [0, 1, 17]
    rows, owner = [], []
    for e in range(len(G)):
        if G[e] == 0:
            continue
        t = np.arange(1, G[e] + 1, dtype=np.float32) / np.float32(G[e])
        d = to[e] - frm[e]
        # t * d is exact in FP64; one rounding to FP32 after adding from
        rows.append((t[:, None].astype(np.float64) * d + frm[e].astype(np.float64)).astype(np.float32))
        owner.append(np.full(G[e], e))
    Q, own = np.concatenate(rows), np.concatenate(owner)
    _, cc = api.check_configs(b, sc, torch.from_numpy(Q).cuda(), clearance="esdf")
    cc = cc.cpu().numpy()
    rcc = ref.esdf_min_clearance(Q)
    err = np.abs(cc - rcc).max()
    print(f"config ESDF clearance: max |ours - reference| = {err:.2e} m over {len(Q)} configs, "
          f"below 1000: {np.mean(rcc < 999):.2f}")
    assert err < 1e-5
    expect = np.full(len(G), np.finfo(np.float32).max, np.float32)
    np.minimum.at(expect, own, cc)
    rv, _, _ = ref.check_edges(frm, to, G)
    f, t_, g = (torch.from_numpy(x).cuda() for x in (frm, to, G))
    p = api.EdgeEvalParams(compute_clearance=True)
    for persistent in (True, False):
        v, _, clr = api.check_edges(b, sc, f, t_, samples=g, params=p, persistent=persistent)
        np.testing.assert_array_equal(v.cpu().numpy(), rv, err_msg=f"persistent={persistent}")
        clr = clr.cpu().numpy()
        assert np.array_equal(clr.view(np.uint32), expect.view(np.uint32)), (
            persistent, np.abs(clr - expect).max())


def test_costs_with_masks(case):
    asset, obbs, esdf, b, sc, ref, _, masks = case
    rng = np.random.default_rng(5)
    B, T = 32, 24
    s, e = workloads.uniform_configs(rng, asset, B), workloads.uniform_configs(rng, asset, B)
    a = np.linspace(0.0, 1.0, T, dtype=np.float32)[None, :, None]
    q = (s[:, None, :] + a * (e - s)[:, None, :]).astype(np.float32)
    w, wm, sm = 2.0, 0.05, 0.01
    p = api.CostParams(collision_cost_weight=w, world_collision_margin=wm, self_collision_margin=sm)
    wp, _, _ = api.traj_cost(b, sc, torch.from_numpy(q).cuda(), p, want_grad=False)
    ours = wp.cpu().numpy().reshape(-1)
    rsc, _, _ = ref.chomp(q.transpose(0, 2, 1), w, wm, sm, grad=False)
    rref = rsc[:, 0, :].reshape(-1)
    rel = np.abs(ours - rref) / np.maximum(np.abs(rref), 1.0)
    om = oracle.OracleModel(b, *obbs, esdf=esdf)
    om.set_masks(masks["sphere_acm_mask"], masks["sphere_obb_acm_mask"], masks["sphere_obb_acm_mask_approx"])
    c64 = om.state_cost(q.reshape(-1, q.shape[2]), w, wm, sm)
    rel64 = np.abs(ours - c64) / np.maximum(np.abs(c64), 1.0)
    print(f"masked waypoint cost: max rel diff vs reference {rel.max():.2e}, vs fp64 {rel64.max():.2e}, "
          f"active {(c64 > 0).mean():.2f}")
    assert (c64 > 0).mean() > 0.2
    assert rel.max() < 1e-3 and rel64.max() < COST_REL_TOL
    r = q.transpose(0, 2, 1).copy()    # the same waypoints as rollouts [R, D, T]
    rc = api.rollout_costs(b, sc, torch.from_numpy(r).cuda(), p, broadcast_d=True).cpu().numpy()
    theirs, _ = ref.stomp(r, w, wm, sm)
    relr = np.abs(rc - theirs) / np.maximum(np.abs(theirs), 1.0)
    print(f"masked rollout cost: max rel diff vs reference stomp kernel {relr.max():.2e}")
    assert relr.max() < 1e-3
    # the mixed batch's trajectory branch reads the same masks: bitwise equal
    batch = api.MixedBatch(b, 0, 0, 2, 2 * T, T)
    qt = [torch.from_numpy(q[i]).cuda() for i in (0, 7)]
    outs = [batch.add_trajectory(x) for x in qt]
    batch.launch(sc, api.EdgeEvalParams(), p)
    torch.cuda.synchronize()
    for x, (bw, bt, bg) in zip(qt, outs):
        w1, t1, g1 = api.traj_cost(b, sc, x[None], p)
        assert torch.equal(bw.view(torch.int32), w1[0].view(torch.int32))
        assert torch.equal(bg.view(torch.int32), g1[0].view(torch.int32))
    batch.close()


def test_cost_gradient_with_obb_masks(case):
    asset, obbs, _, b, _, _, _, masks = case
    sc = SceneTensors(*obbs, sphere_obb_acm_mask=masks["sphere_obb_acm_mask"])
    rng = np.random.default_rng(6)
    q = workloads.uniform_configs(rng, asset, 64).reshape(8, 8, -1)
    w, wm, sm = 2.0, 0.08, 0.01
    p = api.CostParams(collision_cost_weight=w, world_collision_margin=wm, self_collision_margin=sm)
    _, _, g = api.traj_cost(b, sc, torch.from_numpy(q).cuda(), p)
    ours = g.cpu().numpy().reshape(-1, q.shape[2])
    om = oracle.OracleModel(b, *obbs)
    om.set_masks(None, masks["sphere_obb_acm_mask"], None)
    flat = q.reshape(-1, q.shape[2])
    fd = om.state_cost_fd_grad(flat, w, wm, sm, h=1e-6)
    assert_gradient_vs_fd(ours, fd, om.kink_distance(flat, wm, sm), "masked gradient")
