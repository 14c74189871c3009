"""GPU parity of the mixed-request batch (ps_batch_*): one graph launch over
many uneven edge requests and trajectory requests must give, per request,
the same bits as the per-request calls (which are themselves pinned to the
reference kernels and the FP64 oracle in test_gpu_parity.py), and edge
verdicts bit-exact against the reference kernels directly."""
import numpy as np
import pytest
from conftest import COST_REL_TOL, assert_gradient_vs_fd
import torch

import oracle
from prismplan_b200 import api, workloads
from prismplan_b200._lib import PrismError
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu


def _cost_params(wl, smooth=0.0):
    return api.CostParams(collision_cost_weight=wl["w"], world_collision_margin=wl["eps"],
                          self_collision_margin=wl["self_margin"], smoothness_weight=smooth, delta_t=0.1)


def _fill(batch, wl, n_req=None, n_traj=None, given_every=2):
    """Queue the workload's edge requests (every `given_every`-th with explicit
    sample counts, the rest by the L-inf rule) and trajectories."""
    frm = torch.from_numpy(wl["from"]).cuda()
    to = torch.from_numpy(wl["to"]).cuda()
    G = torch.from_numpy(wl["G"]).cuda()
    reqs, off = [], 0
    for i, k in enumerate(wl["edge_splits"][:n_req]):
        sl = slice(off, off + k)
        smp = G[sl] if i % given_every == 0 else None
        v, c = batch.add_edges(frm[sl], to[sl], smp)
        reqs.append((sl, smp, v, c))
        off += k
    trajs = []
    for q in wl["trajectories"][:n_traj]:
        qt = torch.from_numpy(q).cuda()
        trajs.append((qt,) + batch.add_trajectory(qt))
    return frm, to, reqs, trajs


def _check_against_calls(b, sc, frm, to, reqs, trajs, ep, cp):
    for sl, smp, v, c in reqs:
        v1, c1, _ = api.check_edges(b, sc, frm[sl], to[sl], samples=smp, params=ep, persistent=False)
        assert torch.equal(v, v1)
        assert torch.equal(c.view(torch.int32), c1.view(torch.int32))
    for qt, wp, tc, g in trajs:
        wp1, tc1, g1 = api.traj_cost(b, sc, qt[None], cp)
        assert torch.equal(wp.view(torch.int32), wp1[0].view(torch.int32))
        assert torch.equal(tc.view(torch.int32), tc1.view(torch.int32))
        assert torch.equal(g.view(torch.int32), g1[0].view(torch.int32))


# Launch shapes: the default (the edge queue and the waypoint kernel side by
# side) and the one work-queue kernel (layout 1) at both block widths, with
# all or some of its warps taking waypoint groups.
SHAPES = [None, (1, 128, 4), (1, 256, 2)]


def _shape(batch, shape):
    if shape is not None:
        batch.set_shape(layout=shape[0], work_threads=shape[1], work_cost_warps=shape[2])


@pytest.fixture(scope="module")
def w5():
    wl = workloads.workload(5, scale=1.0 / 4)
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"], *wl["esdf"])
    return wl, b, sc


@pytest.mark.parametrize("shape", SHAPES)
def test_batch_equals_per_request_calls(w5, shape):
    wl, b, sc = w5
    nw = sum(len(q) for q in wl["trajectories"])
    batch = api.MixedBatch(b, len(wl["edge_splits"]), len(wl["from"]), len(wl["trajectories"]), nw, 128)
    _shape(batch, shape)
    frm, to, reqs, trajs = _fill(batch, wl)
    ep = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    cp = _cost_params(wl, smooth=0.5)
    batch.launch(sc, ep, cp)
    torch.cuda.synchronize()
    _check_against_calls(b, sc, frm, to, reqs, trajs, ep, cp)
    # replay with a different mix (fewer requests, same capture)
    batch.clear()
    frm, to, reqs, trajs = _fill(batch, wl, n_req=len(wl["edge_splits"]) // 2, n_traj=3, given_every=3)
    batch.launch(sc, ep, cp)
    torch.cuda.synchronize()
    _check_against_calls(b, sc, frm, to, reqs, trajs, ep, cp)
    batch.close()


@pytest.mark.parametrize("shape", SHAPES)
def test_batch_edges_bitexact_vs_reference(w5, shape):
    wl, b, sc = w5
    ref = oracle.RefKernels(b, *wl["obbs"], esdf=wl["esdf"])
    n = len(wl["from"])
    batch = api.MixedBatch(b, len(wl["edge_splits"]), n, 0, 0, 0)
    _shape(batch, shape)
    frm, to, reqs, _ = _fill(batch, wl, n_traj=0, given_every=1)
    batch.launch(sc, api.EdgeEvalParams(), api.CostParams())
    torch.cuda.synchronize()
    v = torch.cat([r[2] for r in reqs]).cpu().numpy()
    c = torch.cat([r[3] for r in reqs]).cpu().numpy()
    rv, rc, _ = ref.check_edges(wl["from"], wl["to"], wl["G"])
    np.testing.assert_array_equal(v, rv)
    assert np.array_equal(c.view(np.uint32), rc.view(np.uint32))
    assert 0.02 < v.mean() < 0.98
    batch.close()


@pytest.mark.parametrize("shape", SHAPES)
def test_batch_fast_path_panda(w5, shape):
    """Panda-like chain (the single-frame fast edge kernel) with OBBs only."""
    wl2 = workloads.workload(2, scale=1.0 / 16)
    wl3 = workloads.workload(3, scale=1.0 / 16)
    b = RobotModelBuilder.from_asset(wl2["asset"]).build()
    sc = SceneTensors(*wl2["obbs"])
    ref = oracle.RefKernels(b, *wl2["obbs"])
    rng = np.random.default_rng(5)
    n = len(wl2["from"])
    splits, left = [], n
    while left:
        k = min(left, int(rng.integers(1, 300)))
        splits.append(k)
        left -= k
    wl = {"from": wl2["from"], "to": wl2["to"], "G": wl2["G"], "edge_splits": splits,
          "trajectories": list(wl3["q"]), "w": wl3["w"], "eps": wl3["eps"], "self_margin": wl3["self_margin"]}
    nw = sum(len(q) for q in wl["trajectories"])
    batch = api.MixedBatch(b, len(splits), n, len(wl["trajectories"]), nw, 64)
    _shape(batch, shape)
    frm, to, reqs, trajs = _fill(batch, wl, given_every=1)
    ep = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    cp = _cost_params(wl)
    batch.launch(sc, ep, cp)
    torch.cuda.synchronize()
    _check_against_calls(b, sc, frm, to, reqs, trajs, ep, cp)
    v = torch.cat([r[2] for r in reqs]).cpu().numpy()
    rv, _, _ = ref.check_edges(wl2["from"], wl2["to"], wl2["G"])
    np.testing.assert_array_equal(v, rv)
    batch.close()


def test_batch_trilinear_esdf_vs_fp64(w5):
    wl, b, _ = w5
    sc = SceneTensors(*wl["obbs"], *wl["esdf"], esdf_mode=1)
    om = oracle.OracleModel(b, *wl["obbs"], esdf=wl["esdf"], esdf_mode=1)
    trajs = wl["trajectories"][:6]
    nw = sum(len(q) for q in trajs)
    batch = api.MixedBatch(b, 0, 0, len(trajs), nw, 128)
    outs = [batch.add_trajectory(torch.from_numpy(q).cuda()) for q in trajs]
    batch.launch(sc, api.EdgeEvalParams(), _cost_params(wl))
    torch.cuda.synchronize()
    q = np.concatenate(trajs)
    wp = torch.cat([o[0] for o in outs]).cpu().numpy()
    g = torch.cat([o[2] for o in outs]).cpu().numpy()
    c64 = om.state_cost(q, wl["w"], wl["eps"], wl["self_margin"])
    rel = np.abs(wp - c64) / np.maximum(np.abs(c64), 1.0)
    print(f"trilinear ESDF cost: max rel err vs fp64 = {rel.max():.2e}, active = {(c64 > 0).mean():.2f}")
    assert rel.max() < COST_REL_TOL
    # trilinear cells put a gradient kink on every 5 mm voxel face: a smaller
    # step keeps most waypoints clear of one
    fd = om.state_cost_fd_grad(q, wl["w"], wl["eps"], wl["self_margin"], h=1e-7)
    kink = om.kink_distance(q, wl["eps"], wl["self_margin"])
    assert_gradient_vs_fd(g, fd, kink, "trilinear ESDF gradient", h=1e-7)
    batch.close()


def test_batch_tune_keeps_results(w5):
    wl, b, sc = w5
    nw = sum(len(q) for q in wl["trajectories"])
    batch = api.MixedBatch(b, len(wl["edge_splits"]), len(wl["from"]), len(wl["trajectories"]), nw, 128)
    frm, to, reqs, trajs = _fill(batch, wl)
    ep = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    cp = _cost_params(wl)
    t = batch.tune(sc, ep, cp)
    assert t["traj_threads"] in (128, 256) and 0.0 < t["edge_share"] <= 1.0 and t["best_ms"] > 0.0
    assert t["layout"] in (0, 1) and t["work_threads"] in (128, 256)
    print(f"tuned batch shape: {t}")
    batch.launch(sc, ep, cp)
    torch.cuda.synchronize()
    _check_against_calls(b, sc, frm, to, reqs, trajs, ep, cp)
    batch.close()


def test_batch_argument_errors(w5):
    wl, b, sc = w5
    batch = api.MixedBatch(b, 1, 4, 1, 64, 64)
    with pytest.raises(PrismError):
        batch.set_shape(layout=2)
    with pytest.raises(PrismError):
        batch.set_shape(layout=1, work_threads=96)
    with pytest.raises(PrismError):
        batch.set_shape(edge_share=0.0)
    with pytest.raises(PrismError):
        batch.set_shape(layout=1, work_threads=128, work_cost_warps=5)
    q = torch.zeros((65, b.n_dof), device="cuda")
    with pytest.raises(PrismError):
        batch.add_trajectory(q)                        # longer than max_traj_len
    batch.add_trajectory(q[:32])
    with pytest.raises(PrismError):
        batch.add_trajectory(q[:8])                    # too many trajectory requests
    e = torch.zeros((5, b.n_dof), device="cuda")
    with pytest.raises(PrismError):
        batch.add_edges(e, e)                          # edge capacity exceeded
    batch.add_edges(e[:4], e[:4])
    with pytest.raises(PrismError):
        batch.launch(sc, api.EdgeEvalParams(compute_clearance=True), api.CostParams())
    batch.launch(sc, api.EdgeEvalParams(), api.CostParams())
    torch.cuda.synchronize()
    batch.close()


@pytest.mark.parametrize("shape", SHAPES)
def test_batch_edge_cases(w5, shape):
    """Empty launch, G in {0, 1, 33}, a one-waypoint trajectory, replay after
    clear: each equals its per-request call."""
    wl, b, sc = w5
    batch = api.MixedBatch(b, 4, 64, 4, 256, 128)
    _shape(batch, shape)
    ep = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    cp = _cost_params(wl, smooth=0.5)
    batch.launch(sc, ep, cp)                       # no requests at all
    torch.cuda.synchronize()
    frm = torch.from_numpy(wl["from"][:6]).cuda()
    to = torch.from_numpy(wl["to"][:6]).cuda()
    G = torch.tensor([0, 1, 33, 2, 600, 31], dtype=torch.int32, device="cuda")
    v, c = batch.add_edges(frm, to, G)
    q1 = torch.from_numpy(wl["trajectories"][0][:1]).cuda()   # T = 1
    wp, tc, g = batch.add_trajectory(q1)
    batch.launch(sc, ep, cp)
    torch.cuda.synchronize()
    v1, c1, _ = api.check_edges(b, sc, frm, to, samples=G, params=ep, persistent=False)
    assert torch.equal(v, v1) and torch.equal(c.view(torch.int32), c1.view(torch.int32))
    wp1, tc1, g1 = api.traj_cost(b, sc, q1[None], cp)
    assert torch.equal(wp.view(torch.int32), wp1[0].view(torch.int32))
    assert torch.equal(tc.view(torch.int32), tc1.view(torch.int32))
    assert torch.equal(g.view(torch.int32), g1[0].view(torch.int32))
    batch.clear()
    batch.launch(sc, ep, cp)                       # empty again after clear
    torch.cuda.synchronize()
    batch.close()
    with pytest.raises(RuntimeError):
        batch.launch(sc, ep, cp)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("broadcast", [False, True])
def test_batch_rollouts_equal_rollout_costs(w5, broadcast, shape):
    """STOMP rollout requests (reference layout [R, D, T]) share the launch
    with edge and trajectory requests; their state costs equal
    ps_rollout_costs bit for bit, and the other requests are unchanged."""
    wl, b, sc = w5
    rng = np.random.default_rng(55)
    trajs = wl["trajectories"][:3]
    rolls = []
    for q in trajs[:2]:   # noisy copies of a trajectory, reference layout
        r = q[None].transpose(0, 2, 1) + rng.normal(0.0, 0.05, (9,) + q.T.shape).astype(np.float32)
        rolls.append(torch.from_numpy(np.ascontiguousarray(r, np.float32)).cuda())
    nw = sum(len(q) for q in trajs) + sum(r.shape[0] * r.shape[2] for r in rolls)
    n_req = 4
    n_e = sum(wl["edge_splits"][:n_req])
    batch = api.MixedBatch(b, n_req, n_e, 3 + len(rolls), nw, 128)
    _shape(batch, shape)
    r_out = [batch.add_rollouts(rolls[0], broadcast_d=broadcast)]
    frm, to, reqs, tr = _fill(batch, wl, n_req=n_req, n_traj=3)
    r_out.append(batch.add_rollouts(rolls[1], broadcast_d=broadcast))
    ep = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    cp = _cost_params(wl, 1.0)
    batch.launch(sc, ep, cp)
    torch.cuda.synchronize()
    for r, out in zip(rolls, r_out):
        ref = api.rollout_costs(b, sc, r, cp, broadcast_d=broadcast)
        assert out.shape == ref.shape
        assert torch.equal(out.view(torch.int32), ref.view(torch.int32))
    assert float(r_out[0].max()) > 0.0
    _check_against_calls(b, sc, frm, to, reqs, tr, ep, cp)
    batch.close()
