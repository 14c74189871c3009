"""GPU: every kernel fails closed when its bounded model-staging wait gives up.

The wait limit is set to 0 polls through ps_model_set_wait_limit, so every
launch gives up at once (the copy in flight is still drained, bounded): no
fault, no hang. Each path must then report nothing as free: configurations
in collision, edges invalid with cost FLT_MAX, costs and gradients NaN, and
the statuses PS_ETIMEOUT. Restoring the limit gives the normal results back.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from prismplan_b200 import _lib, api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu

FLT_MAX = np.finfo(np.float32).max


@pytest.fixture()
def setup():
    wl = workloads.workload(2, scale=1.0 / 16)   # 4096 edges
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    frm = torch.from_numpy(wl["from"]).cuda()
    to = torch.from_numpy(wl["to"]).cuda()
    yield b, sc, frm, to, wl
    _lib.check(_lib.load().ps_model_set_wait_limit(b.handle, -1))


def _poll(b):
    code = C.c_int(-1)
    _lib.check(_lib.load().ps_model_poll_status(b.handle, C.byref(code)))
    return code.value


def _give_up(b, on):
    _lib.check(_lib.load().ps_model_set_wait_limit(b.handle, 0 if on else -1))


@pytest.mark.parametrize("check_self", [False, True])
def test_configs_fail_closed(setup, check_self):
    b, sc, frm, _, _ = setup
    q = frm[:1000].contiguous()
    hit_ok, _ = api.check_configs(b, sc, q, clearance="obb", check_self=check_self)
    if not check_self:   # (this synthetic chain self-collides almost everywhere)
        assert 0.0 < float(hit_ok.float().mean()) < 1.0
    assert _poll(b) == _lib.PS_OK
    _give_up(b, True)
    hit, clr = api.check_configs(b, sc, q, clearance="obb", check_self=check_self)
    torch.cuda.synchronize()
    assert bool((hit == 1).all())
    assert bool(torch.isnan(clr).all())
    assert _poll(b) == _lib.PS_ETIMEOUT
    assert _poll(b) == _lib.PS_OK   # polling clears the latch
    _give_up(b, False)
    hit2, _ = api.check_configs(b, sc, q, clearance="obb", check_self=check_self)
    assert torch.equal(hit2, hit_ok)
    assert _poll(b) == _lib.PS_OK


def _static(b, sc, frm, to, p):
    E = frm.shape[0]
    v = torch.full((E,), 7, dtype=torch.uint8, device="cuda")
    c = torch.empty(E, dtype=torch.float32, device="cuda")
    k = torch.empty(E, dtype=torch.float32, device="cuda")
    pc = p.to_c()
    view = sc.view()
    _lib.check(_lib.load().ps_check_edges_static(b.handle, C.byref(view), frm.data_ptr(), to.data_ptr(), None, E,
                                                 C.byref(pc), v.data_ptr(), c.data_ptr(), k.data_ptr(), None))
    return v, c


@pytest.mark.parametrize("path", ["persistent", "plain", "static"])
@pytest.mark.parametrize("check_self", [False, True])
def test_edges_fail_closed(setup, path, check_self):
    b, sc, frm, to, wl = setup
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600, check_self=check_self)
    ws = api.edges_workspace(frm.shape[0]) if path == "persistent" else None

    def run():
        if path == "static":
            return _static(b, sc, frm, to, p)
        v, c, _ = api.check_edges(b, sc, frm, to, params=p, persistent=path == "persistent", workspace=ws)
        return v, c

    v_ok, _ = run()
    torch.cuda.synchronize()
    if not check_self:   # (this synthetic chain self-collides on almost every edge)
        assert float(v_ok.float().mean()) > 0.02
    _give_up(b, True)
    v, c = run()
    torch.cuda.synchronize()
    v, c = v.cpu().numpy(), c.cpu().numpy()
    has_samples = wl["G"] > 0
    assert not np.any(v[has_samples] == 1), "an unchecked edge was reported free"
    assert np.all(c[has_samples] == FLT_MAX)
    assert _poll(b) == _lib.PS_ETIMEOUT
    if path == "persistent":
        assert api.edges_status(ws) == _lib.PS_ETIMEOUT
    elif path == "static":
        assert api.edges_status(None) == _lib.PS_ETIMEOUT
    _give_up(b, False)
    v2, _ = run()
    torch.cuda.synchronize()
    assert torch.equal(v2, v_ok)
    if path == "persistent":
        assert api.edges_status(ws) == _lib.PS_OK


@pytest.mark.parametrize("want_grad", [True, False])
def test_costs_fail_closed(setup, want_grad):
    b, sc, _, _, _ = setup
    w3 = workloads.workload(3, scale=1.0 / 64)
    q = torch.from_numpy(w3["q"]).cuda()
    p = api.CostParams(collision_cost_weight=w3["w"], world_collision_margin=w3["eps"],
                       self_collision_margin=w3["self_margin"], smoothness_weight=1.0, delta_t=w3["delta_t"])
    b3 = RobotModelBuilder.from_asset(w3["asset"]).build()
    sc3 = SceneTensors(*w3["obbs"])
    wp_ok, tc_ok, _ = api.traj_cost(b3, sc3, q, p, want_grad=want_grad)
    torch.cuda.synchronize()
    assert bool(torch.isfinite(wp_ok).all())
    _lib.check(_lib.load().ps_model_set_wait_limit(b3.handle, 0))
    try:
        wp, tc, g = api.traj_cost(b3, sc3, q, p, want_grad=want_grad)
        torch.cuda.synchronize()
        assert bool(torch.isnan(wp).all()) and bool(torch.isnan(tc).all())
        if want_grad:
            assert bool(torch.isnan(g).all())
        assert _poll(b3) == _lib.PS_ETIMEOUT
        rc = api.rollout_costs(b3, sc3, q.transpose(1, 2).contiguous(), p)
        torch.cuda.synchronize()
        assert bool(torch.isnan(rc).all())
        assert _poll(b3) == _lib.PS_ETIMEOUT
    finally:
        _lib.check(_lib.load().ps_model_set_wait_limit(b3.handle, -1))
    wp2, tc2, _ = api.traj_cost(b3, sc3, q, p, want_grad=want_grad)
    assert torch.equal(wp2, wp_ok) and torch.equal(tc2, tc_ok)


@pytest.mark.parametrize("layout", [0, 1, 2])
def test_batch_fail_closed(setup, layout):
    b, sc, frm, to, _ = setup
    E = frm.shape[0]
    w3 = workloads.workload(3, scale=1.0 / 64)
    q = torch.from_numpy(w3["q"][:, :, :]).cuda()
    batch = api.MixedBatch(b, 4, E, 4, 4 * q.shape[1], q.shape[1])
    batch.set_shape(layout=min(layout, 1), work_cost_warps=2 if layout == 2 else None)   # 2: some warps edges only
    outs = [batch.add_edges(frm[i::4], to[i::4]) for i in range(4)]
    touts = [batch.add_trajectory(q[i].contiguous()) for i in range(4)]
    ep = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    cp = api.CostParams(collision_cost_weight=w3["w"], world_collision_margin=w3["eps"],
                        self_collision_margin=w3["self_margin"])
    batch.launch(sc, ep, cp)
    assert batch.status() == _lib.PS_OK
    v_ok = torch.cat([o[0] for o in outs]).cpu().numpy()
    assert v_ok.mean() > 0.02
    _give_up(b, True)
    batch.launch(sc, ep, cp)
    assert batch.status() == _lib.PS_ETIMEOUT
    v = torch.cat([o[0] for o in outs]).cpu().numpy()
    assert not np.any(v == 1)
    for wp, tc, g in touts:
        assert bool(torch.isnan(wp).all()) and bool(torch.isnan(tc).all()) and bool(torch.isnan(g).all())
    _give_up(b, False)
    assert _poll(b) == _lib.PS_ETIMEOUT
    batch.close()
