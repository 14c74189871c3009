"""GPU: the standalone autotuners (ps_tune_edges, ps_tune_configs) pick a
launch shape by timing candidates on the caller's inputs; results do not
depend on the shape, so the tuned calls must equal the default ones bit for
bit."""
import numpy as np
import pytest
import torch

from prismplan_b200 import api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu


def test_tune_edges_keeps_results():
    wl = workloads.workload(2, scale=0.6)   # enough edges for the probe to be a candidate
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    frm, to = torch.from_numpy(wl["from"]).cuda(), torch.from_numpy(wl["to"]).cuda()
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    v0, c0, _ = api.check_edges(b, sc, frm, to, params=p)
    tuned, info = api.tune_edges(b, sc, frm, to, params=p)
    print("edge tuning:", info)
    assert info["candidates"] >= 7
    assert 0.0 < info["best_ms"] <= info["default_ms"]
    assert tuned.probe in (1, 2) and 1 <= tuned.queue_blocks_per_sm <= 8 and tuned.grab in (0, 8, 32)
    v1, c1, _ = api.check_edges(b, sc, frm, to, params=tuned)
    assert torch.equal(v0, v1) and torch.equal(c0.view(torch.int32), c1.view(torch.int32))
    for probe in (1, 2):   # every forced shape gives the same bits
        q = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600, probe=probe, queue_blocks_per_sm=2, grab=3)
        v2, c2, _ = api.check_edges(b, sc, frm, to, params=q)
        assert torch.equal(v0, v2) and torch.equal(c0.view(torch.int32), c2.view(torch.int32))


def test_tune_configs_keeps_results():
    wl = workloads.workload(1)
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    q = torch.from_numpy(np.tile(wl["q"], (16, 1))).cuda()
    h0, c0 = api.check_configs(b, sc, q, clearance="obb")
    k, info = api.tune_configs(b, sc, q, clearance="obb")
    print("config tuning:", info)
    assert info["candidates"] == 7 and 1 <= k <= 12
    assert 0.0 < info["best_ms"] <= info["default_ms"]
    h1, c1 = api.check_configs(b, sc, q, clearance="obb", blocks_per_sm=k)
    assert torch.equal(h0, h1) and torch.equal(c0.view(torch.int32), c1.view(torch.int32))
