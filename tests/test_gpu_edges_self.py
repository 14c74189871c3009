"""Edge checks with the self check (check_self, edge_eval.cuh:40 and :128):
every edge path (persistent, plain, static, mixed batch) against the
reference's evaluate_edges_batch run with check_self on the same inputs, bit
for bit, on the reference's Panda where a share of the edges is free of the
scene but not of itself."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from conftest import golden_asset
from prismplan_b200 import _lib, api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(golden):
    asset, _ = golden_asset(golden, "panda")
    rng = np.random.default_rng(2024)
    obbs = workloads.random_obbs(rng, 8)
    b = RobotModelBuilder.from_asset(asset).build()
    sc = SceneTensors(*obbs)
    frm, to, G = workloads.edge_batch(rng, asset, 3000, step=0.02, max_samples=300)
    G[:7] = [0, 1, 15, 16, 17, 32, 33]   # zero samples, the start-sample rule (G % 16) and chunk edges
    ref = oracle.RefKernels(b, *obbs)
    return asset, obbs, b, sc, frm, to, G, ref


def _static(b, sc, frm, to, G, p):
    E = frm.shape[0]
    v = torch.empty(E, dtype=torch.uint8, device="cuda")
    c = torch.empty(E, dtype=torch.float32, device="cuda")
    k = torch.empty(E, dtype=torch.float32, device="cuda")
    pc = p.to_c()
    view = sc.view()
    _lib.check(_lib.load().ps_check_edges_static(b.handle, C.byref(view), frm.data_ptr(), to.data_ptr(),
                                                 G.data_ptr(), E, C.byref(pc), v.data_ptr(), c.data_ptr(),
                                                 k.data_ptr(), None))
    return v, c


def test_edges_self_bitexact_vs_reference(case):
    asset, obbs, b, sc, frm, to, G, ref = case
    rv_scene, _, _ = ref.check_edges(frm, to, G, check_self=False)
    rv, rc, _ = ref.check_edges(frm, to, G, check_self=True)
    only_self = (rv_scene == 1) & (rv == 0)
    print(f"edges: {len(G)}, free of the scene {rv_scene.mean():.3f}, free {rv.mean():.3f}, "
          f"invalid by self only {only_self.sum()}")
    assert only_self.sum() > 20 and rv.sum() > 20
    f, t, g = (torch.from_numpy(x).cuda() for x in (frm, to, G))
    p = api.EdgeEvalParams(check_self=True)
    outs = {
        "persistent": api.check_edges(b, sc, f, t, samples=g, params=p)[:2],
        "plain": api.check_edges(b, sc, f, t, samples=g, params=p, persistent=False)[:2],
        "static": _static(b, sc, f, t, g, p),
    }
    for name, (v, c) in outs.items():
        v, c = v.cpu().numpy(), c.cpu().numpy()
        np.testing.assert_array_equal(v, rv, err_msg=name)
        assert np.array_equal(c.view(np.uint32), rc.view(np.uint32)), name
    # without the self check nothing changes
    v0, c0, _ = api.check_edges(b, sc, f, t, samples=g, params=api.EdgeEvalParams(check_self=False))
    np.testing.assert_array_equal(v0.cpu().numpy(), rv_scene)


def test_edges_self_with_margin(case):
    """A collision margin widens the scene spheres only: the self pairs of
    two_phase_cc take none (two_phase_cc.cuh:109-131)."""
    asset, obbs, b, sc, frm, to, G, ref = case
    n = 1200
    rv, rc, _ = ref.check_edges(frm[:n], to[:n], G[:n], margin=0.01, check_self=True)
    rv0, _, _ = ref.check_edges(frm[:n], to[:n], G[:n], margin=0.0, check_self=True)
    assert (rv != rv0).any()
    f, t, g = (torch.from_numpy(x[:n]).cuda() for x in (frm, to, G))
    p = api.EdgeEvalParams(check_self=True, collision_margin=0.01)
    for persistent in (True, False):
        v, c, _ = api.check_edges(b, sc, f, t, samples=g, params=p, persistent=persistent)
        np.testing.assert_array_equal(v.cpu().numpy(), rv, err_msg=f"persistent={persistent}")
        assert np.array_equal(c.cpu().numpy().view(np.uint32), rc.view(np.uint32))


def test_batch_edges_with_self(case):
    asset, obbs, b, sc, frm, to, G, ref = case
    p = api.EdgeEvalParams(check_self=True)
    n = len(G)
    batch = api.MixedBatch(b, 3, n, 0, 0, 0)
    cuts = [0, 700, 1900, n]
    f, t, g = (torch.from_numpy(x).cuda() for x in (frm, to, G))
    outs = [batch.add_edges(f[cuts[i]:cuts[i + 1]], t[cuts[i]:cuts[i + 1]], g[cuts[i]:cuts[i + 1]])
            for i in range(3)]
    batch.launch(sc, p, api.CostParams())
    torch.cuda.synchronize()
    v = torch.cat([o[0] for o in outs]).cpu().numpy()
    c = torch.cat([o[1] for o in outs]).cpu().numpy()
    rv, rc, _ = ref.check_edges(frm, to, G, check_self=True)
    np.testing.assert_array_equal(v, rv)
    assert np.array_equal(c.view(np.uint32), rc.view(np.uint32))
    batch.close()


def test_self_pass_respects_time_budget(case):
    asset, obbs, b, sc, frm, to, G, ref = case
    f, t, g = (torch.from_numpy(x).cuda() for x in (frm, to, G))
    ws = api.edges_workspace(len(G))
    rv, _, _ = ref.check_edges(frm, to, G, check_self=True)
    v, c, _ = api.check_edges(b, sc, f, t, samples=g, workspace=ws,
                              params=api.EdgeEvalParams(check_self=True, time_budget_ms=1e-6))
    torch.cuda.synchronize()
    assert api.edges_status(ws) == _lib.PS_ETIMEOUT
    v = v.cpu().numpy()
    assert not np.any((v == 1) & (rv == 0))   # never free when not shown free


def _without_last_approx_sphere(asset):
    """The asset with its last approximate sphere removed (and the approximate
    self ranges that name it trimmed): that joint keeps its exact spheres but
    has no approximate sphere, so its bound centre cannot be read off one."""
    a = {k: (list(v) if isinstance(v, (list, tuple, np.ndarray)) else v) for k, v in asset.items()}
    na = len(a["approx_sphere_to_joint"])
    last = na - 1
    a["approx_spheres_flat"] = list(a["approx_spheres_flat"][: 4 * last])
    a["approx_sphere_to_joint"] = list(a["approx_sphere_to_joint"][:last])
    r = np.asarray(a["approx_self_cc_ranges_flat"], dtype=np.int64).reshape(-1, 3)
    keep = []
    for i, s, e in r:
        e = min(int(e), last - 1)
        if int(i) != last and int(s) <= e:
            keep.append((int(i), int(s), e))
    a["approx_self_cc_ranges_flat"] = [x for t in keep for x in t]
    return a


def test_self_checks_with_staged_bound_centres(case):
    """The self checks read a joint's bound centre off its first approximate
    sphere when every joint with exact spheres has one on the shared chain, and
    stage every bound centre otherwise. This model takes the second layout. The
    reference's kernels assume one approximate sphere per joint with spheres
    (their approximate pass indexes by joint), so this model is held to the
    FP64 oracle: edges with check_self and the configuration self check may
    differ from it only at contact."""
    asset, obbs, _, sc, frm, to, G, _ = case
    a2 = _without_last_approx_sphere(asset)
    b2 = RobotModelBuilder.from_asset(a2).build()
    om = oracle.OracleModel(b2, *obbs)
    rv, _, _, gap_e, _ = om.check_edges(frm, to, G, check_self=True, early_exit=False, want_gap=True)
    f, t, g = (torch.from_numpy(x).cuda() for x in (frm, to, G))
    v = api.check_edges(b2, sc, f, t, samples=g, params=api.EdgeEvalParams(check_self=True))[0].cpu().numpy()
    ef = np.nonzero(v != rv)[0]
    q = np.concatenate([frm, to])[:2048].astype(np.float32)
    h, _ = api.check_configs(b2, None, torch.from_numpy(q).cuda(), check_self=True)
    om0 = oracle.OracleModel(b2, np.zeros((0, 4)), np.zeros((0, 8)))
    h64, _, gap = om0.check_configs(q, flags=_lib.PS_CHECK_SELF, want_gap=True)
    flips = np.nonzero(h.cpu().numpy() != h64)[0]
    print(f"staged bound centres: edges {len(ef)} flips of {len(G)} (distance to contact {gap_e[ef].tolist()}), "
          f"configurations {len(flips)} of {len(q)} ({gap[flips].tolist()}); edges free {rv.mean():.3f}")
    assert np.all(gap_e[ef] < 1e-5) and np.all(gap[flips] < 1e-5)
    assert 0.0 < rv.mean() < 1.0 and h64.mean() > 0.0
    b2.destroy()
