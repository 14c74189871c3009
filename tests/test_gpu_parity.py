"""GPU parity: the CUDA path (through the C ABI) against PrismPlan's own
kernels (oracle/_ref, built from the reference sources) and the FP64 oracle.

Bars: collision Booleans bit-exact against the reference kernels; sphere
centres bitwise equal to the reference FK; edge validity and cost bit-exact;
clearance within 1e-5 m of the reference and of FP64; costs and gradients
within the relative tolerances stated per test against FP64.
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import COST_REL_TOL, assert_gradient_vs_fd, golden_asset
from prismplan_b200 import api, workloads
from prismplan_b200 import _lib
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors, pack_obbs

pytestmark = pytest.mark.gpu

ASSETS = ("panda", "fetch", "baxter")


def make(asset, obbs, esdf=None, esdf_mode=0):
    b = RobotModelBuilder.from_asset(asset).build()
    sc = SceneTensors(*obbs) if esdf is None else SceneTensors(*obbs, *esdf, esdf_mode=esdf_mode)
    om = oracle.OracleModel(b, *obbs, esdf=esdf, esdf_mode=esdf_mode)
    ref = oracle.RefKernels(b, *obbs, esdf=esdf)
    return b, sc, om, ref


def synthetic_assets():
    return {"panda_like": workloads.panda_like(), "fetch_like": workloads.fetch_like(),
            "baxter_like": workloads.baxter_like(), "generic_chain": workloads.generic_chain()}


# ---------------------------------------------------------------------------
# FK
# ---------------------------------------------------------------------------
def _fk_case(asset, q):
    b = RobotModelBuilder.from_asset(asset).build()
    ref = oracle.RefKernels(b, np.zeros((0, 4)), np.zeros((0, 8)))
    ours = api.fk_spheres(b, torch.from_numpy(q).cuda()).cpu().numpy()
    theirs = ref.fk_spheres(q)
    bad = ours.view(np.uint32) != theirs.view(np.uint32)
    assert not bad.any(), (
        f"{bad.sum()} of {bad.size} coordinates differ; max |d| = {np.abs(ours - theirs).max():.3e}")


@pytest.mark.parametrize("name", ASSETS)
def test_fk_bitwise_vs_reference_assets(golden, name):
    asset, raw = golden_asset(golden, name)
    rng = np.random.default_rng(7)
    lo, hi = np.asarray(asset["joint_lower"]), np.asarray(asset["joint_upper"])
    q = (lo + rng.random((2048, len(lo))) * (hi - lo)).astype(np.float32)
    _fk_case(asset, q)


@pytest.mark.parametrize("name", ["panda_like", "fetch_like", "baxter_like", "generic_chain"])
def test_fk_bitwise_vs_reference_synthetic(name):
    asset = synthetic_assets()[name]
    q = workloads.uniform_configs(np.random.default_rng(3), asset, 2048)
    _fk_case(asset, q)


def test_generic_chain_verdicts_bitexact():
    asset = workloads.generic_chain()
    rng = np.random.default_rng(12)
    obbs = workloads.random_obbs(rng, 24)
    b, sc, om, ref = make(asset, obbs)
    q = workloads.uniform_configs(rng, asset, 4096)
    hit, _ = api.check_configs(b, sc, torch.from_numpy(q).cuda())
    rhit, _ = ref.check_configs(q)
    np.testing.assert_array_equal(hit.cpu().numpy(), rhit)
    assert 0.02 < rhit.mean() < 0.98


def test_fk_close_to_fp64():
    asset = workloads.baxter_like()
    q = workloads.uniform_configs(np.random.default_rng(5), asset, 512)
    b = RobotModelBuilder.from_asset(asset).build()
    om = oracle.OracleModel(b, np.zeros((0, 4)), np.zeros((0, 8)))
    ours = api.fk_spheres(b, torch.from_numpy(q).cuda()).cpu().numpy()
    assert np.abs(ours - om.fk_spheres(q)).max() < 5e-6   # __sinf/__cosf + FP32


# ---------------------------------------------------------------------------
# configuration checks (workload 1 and the reference assets)
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def w1():
    wl = workloads.workload(1)
    b, sc, om, ref = make(wl["asset"], wl["obbs"])
    return wl, b, sc, om, ref


def test_config_verdicts_bitexact_vs_reference(w1):
    wl, b, sc, om, ref = w1
    q = torch.from_numpy(wl["q"]).cuda()
    hit, clr = api.check_configs(b, sc, q, clearance="obb")
    hit_nc, _ = api.check_configs(b, sc, q)
    rhit, _ = ref.check_configs(wl["q"])
    ours = hit.cpu().numpy()
    np.testing.assert_array_equal(ours, rhit)
    np.testing.assert_array_equal(hit_nc.cpu().numpy(), rhit)
    assert 0.02 < ours.mean() < 0.98
    # flips against FP64 are only allowed at contact (distance to contact reported)
    h64, _, gap = om.check_configs(wl["q"])
    flips = np.nonzero(h64 != ours)[0]
    assert len(flips) == 0 or np.abs(gap[flips]).max() < 1e-5, gap[flips]


@pytest.mark.parametrize("margin", [0.0, 0.01, -0.005])
def test_config_verdicts_with_margin(w1, margin):
    wl, b, sc, om, ref = w1
    q = wl["q"][:1024]
    hit, _ = api.check_configs(b, sc, torch.from_numpy(q).cuda(), collision_margin=margin)
    rhit, _ = ref.check_configs(q, margin)
    np.testing.assert_array_equal(hit.cpu().numpy(), rhit)


def test_near_tie_decisions_bitexact(w1):
    """Margins set to each configuration's own FP64 distance to contact put
    the decisive pair on the rounding boundary: the exact fallback must
    reproduce the reference's FP32 decision bit for bit."""
    wl, b, sc, om, ref = w1
    q = wl["q"][:96]
    _, _, gap = om.check_configs(q, flags=_lib.PS_NO_GATE)
    n_true = 0
    for i in range(len(q)):
        for k in (-1, 0, 1):
            m = np.float32(gap[i]) if np.isfinite(gap[i]) and abs(gap[i]) < 0.5 else np.float32(0.0)
            m = np.nextafter(m, np.float32(np.inf * k)) if k else m
            one = q[i:i + 1]
            h, _ = api.check_configs(b, sc, torch.from_numpy(one).cuda(), collision_margin=float(m))
            rh, _ = ref.check_configs(one, float(m))
            assert int(h.item()) == int(rh[0]), (i, k, float(m))
            n_true += int(rh[0])
    assert n_true > 0


@pytest.mark.parametrize("name", ASSETS)
def test_config_verdicts_reference_assets(golden, name):
    asset, raw = golden_asset(golden, name)
    for s in range(raw["obb_dims"].shape[0]):
        obbs = pack_obbs(raw["obb_dims"][s], raw["obb_pos"][s], raw["obb_quat"][s])
        b, sc, om, ref = make(asset, obbs)
        q = raw["q"]
        hit, _ = api.check_configs(b, sc, torch.from_numpy(q).cuda())
        rhit, _ = ref.check_configs(q)
        np.testing.assert_array_equal(hit.cpu().numpy(), rhit)
        assert (rhit.astype(bool) == raw["in_collision"][s]).mean() > 0.97


def test_obb_clearance_vs_reference_and_fp64(w1):
    wl, b, sc, om, ref = w1
    q = wl["q"][:2048]
    _, clr = api.check_configs(b, sc, torch.from_numpy(q).cuda(), clearance="obb")
    ours = clr.cpu().numpy()
    rclr = ref.obb_min_clearance(q)
    _, c64, _ = om.check_configs(q, flags=_lib.PS_CLEARANCE_OBB)
    err_ref = np.abs(ours - rclr).max()
    err_64 = np.abs(ours - c64).max()
    print(f"clearance max |ours - reference| = {err_ref:.2e} m, max |ours - fp64| = {err_64:.2e} m")
    assert err_ref < 1e-5 and err_64 < 1e-5


def test_gate_changes_nothing(w1):
    wl, b, sc, om, ref = w1
    q = torch.from_numpy(wl["q"]).cuda()
    g, _ = api.check_configs(b, sc, q)
    ng, _ = api.check_configs(b, sc, q, no_gate=True)
    assert int((g != ng).sum()) == 0


def test_config_edge_cases(w1):
    wl, b, sc, om, ref = w1
    empty = torch.zeros((0, 7), device="cuda")
    h, _ = api.check_configs(b, sc, empty)
    assert h.numel() == 0
    q = torch.from_numpy(wl["q"][:256]).cuda()
    h, c = api.check_configs(b, None, q, clearance="obb")          # empty world
    assert int(h.sum()) == 0 and torch.all(c == 1000.0)
    d, p, en = wl["obbs"]
    off = SceneTensors(d, p, np.zeros_like(en))                    # all boxes disabled
    h, c = api.check_configs(b, off, q, clearance="obb")
    assert int(h.sum()) == 0 and torch.all(c == 1000.0)
    one = SceneTensors(d[:1], p[:1], en[:1])                       # a single box
    h, _ = api.check_configs(b, one, q)
    rb = oracle.RefKernels(b, d[:1], p[:1], en[:1])
    np.testing.assert_array_equal(h.cpu().numpy(), rb.check_configs(wl["q"][:256])[0])
    assert api.check_collision_scene(wl["q"][:8], sc.builder, b).dtype == bool


def test_self_check_vs_oracle(w1):
    wl, b, sc, om, ref = w1
    q = wl["q"][:1024]
    h, _ = api.check_configs(b, None, torch.from_numpy(q).cuda(), check_self=True)
    om0 = oracle.OracleModel(b, np.zeros((0, 4)), np.zeros((0, 8)))
    h64, _, gap = om0.check_configs(q, flags=_lib.PS_CHECK_SELF, want_gap=True)
    flips = np.nonzero(h.cpu().numpy() != h64)[0]
    print(f"self check vs FP64: {len(flips)} flips of {len(q)}; FP64 distance to contact (m) of each: "
          f"{gap[flips].tolist()}")
    assert np.all(gap[flips] < 1e-5), "a self-check flip away from contact"
    assert h64.mean() > 0.0


def test_esdf_nearest_vs_reference():
    asset = workloads.baxter_like()
    rng = np.random.default_rng(11)
    obbs = workloads.random_obbs(rng, 8)
    esdf = workloads.random_esdf(rng, n_vox=64, voxel=0.01)
    b, sc, om, ref = make(asset, obbs, esdf=esdf)
    q = workloads.uniform_configs(rng, asset, 2048)
    hit, _ = api.check_configs(b, sc, torch.from_numpy(q).cuda())
    rhit, _ = ref.check_configs(q)
    np.testing.assert_array_equal(hit.cpu().numpy(), rhit)


# ---------------------------------------------------------------------------
# edges (workload 2)
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def w2():
    wl = workloads.workload(2, scale=1.0 / 32)
    b, sc, om, ref = make(wl["asset"], wl["obbs"])
    return wl, b, sc, om, ref


@pytest.mark.parametrize("persistent", [True, False])
def test_edges_bitexact_vs_reference(w2, persistent):
    wl, b, sc, om, ref = w2
    frm, to, G = wl["from"], wl["to"], wl["G"]
    v, c, _ = api.check_edges(b, sc, torch.from_numpy(frm).cuda(), torch.from_numpy(to).cuda(),
                              samples=torch.from_numpy(G).cuda(), persistent=persistent)
    rv, rc, _ = ref.check_edges(frm, to, G)
    v, c = v.cpu().numpy(), c.cpu().numpy()
    np.testing.assert_array_equal(v, rv)
    assert np.array_equal(c.view(np.uint32), rc.view(np.uint32))
    assert 0.02 < v.mean() < 0.98


def test_edges_linf_rule_matches_given_samples(w2):
    wl, b, sc, om, ref = w2
    frm, to, G = wl["from"], wl["to"], wl["G"]
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    v1, c1, _ = api.check_edges(b, sc, frm, to, params=p)
    v2, c2, _ = api.check_edges(b, sc, frm, to, samples=G)
    assert torch.equal(v1, v2) and torch.equal(c1, c2)


def test_edges_vs_fp64_oracle(w2):
    wl, b, sc, om, ref = w2
    frm, to, G = wl["from"][:512], wl["to"][:512], wl["G"][:512]
    v, _, _ = api.check_edges(b, sc, frm, to, samples=G)
    v64, _, _, gap, _ = om.check_edges(frm, to, G, early_exit=False, want_gap=True)
    flips = np.nonzero(v.cpu().numpy() != v64)[0]
    assert len(flips) == 0 or np.abs(gap[flips]).max() < 1e-5


def test_edges_reference_resolution_rule(w2):
    wl, b, sc, om, ref = w2
    frm, to = wl["from"][:256], wl["to"][:256]
    p = api.EdgeEvalParams(resolution=0.05)
    v, c, _ = api.check_edges(b, sc, frm, to, params=p)
    d = np.linalg.norm((to - frm).astype(np.float32), axis=1).astype(np.float32)
    G = np.clip(np.ceil(d / np.float32(0.05)), 2, 1024).astype(np.int32)
    rv, rc, _ = ref.check_edges(frm, to, G)
    np.testing.assert_array_equal(v.cpu().numpy(), rv)


def test_edges_edge_cases(w2):
    wl, b, sc, om, ref = w2
    frm, to = wl["from"][:64], wl["to"][:64]
    for G in (np.zeros(64, np.int32), np.ones(64, np.int32), np.full(64, 33, np.int32)):
        v, c, _ = api.check_edges(b, sc, frm, to, samples=G)
        rv, rc, _ = ref.check_edges(frm, to, G)
        np.testing.assert_array_equal(v.cpu().numpy(), rv)
    v, _, _ = api.check_edges(b, sc, frm[:0], to[:0], samples=np.zeros(0, np.int32))
    assert v.numel() == 0
    v, _, _ = api.check_edges(b, None, frm, to, samples=np.full(64, 40, np.int32))
    assert int(v.sum()) == 64


def test_edge_bridge_roundtrip(w2):
    wl, b, sc, om, ref = w2
    ev = api.EdgeEvalGpu(7, 256, sc, b)
    p = api.EdgeEvalParams(granularity=40)
    valid, cost, _ = ev.evaluate(wl["from"][:200].reshape(-1), wl["to"][:200].reshape(-1), 200, p)
    rv, rc, _ = ref.check_edges(wl["from"][:200], wl["to"][:200], np.full(200, 40, np.int32))
    np.testing.assert_array_equal(valid, rv)
    with pytest.raises(RuntimeError):
        ev.evaluate(wl["from"], wl["to"], 300, p)
    # later calls of the same size replay a captured graph: feed different edges
    # each time and check every answer against the reference kernels
    for k in range(1, 4):
        sl = slice(200 * k, 200 * (k + 1))
        valid, cost, _ = ev.evaluate(wl["from"][sl].reshape(-1), wl["to"][sl].reshape(-1), 200, p)
        rv, rc, _ = ref.check_edges(wl["from"][sl], wl["to"][sl], np.full(200, 40, np.int32))
        np.testing.assert_array_equal(valid, rv)
        assert np.array_equal(cost.view(np.uint32), rc.view(np.uint32))


def test_edges_graph_capture_replay(w2):
    wl, b, sc, om, ref = w2
    frm = torch.from_numpy(wl["from"]).cuda()
    to = torch.from_numpy(wl["to"]).cuda()
    G = torch.from_numpy(wl["G"]).cuda()
    ws = api.edges_workspace(frm.shape[0])
    out = (torch.empty(frm.shape[0], dtype=torch.uint8, device="cuda"),
           torch.empty(frm.shape[0], device="cuda"), torch.empty(frm.shape[0], device="cuda"))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        api.check_edges(b, sc, frm, to, samples=G, workspace=ws, out=out, stream=s)   # warm-up
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        api.check_edges(b, sc, frm, to, samples=G, workspace=ws, out=out, stream=s)
    for _ in range(3):
        out[0].fill_(7)
        g.replay()
    torch.cuda.synchronize()
    rv, rc, _ = ref.check_edges(wl["from"], wl["to"], wl["G"])
    np.testing.assert_array_equal(out[0].cpu().numpy(), rv)
    del g


def test_model_status_clean(w2):
    wl, b, sc, om, ref = w2
    import ctypes
    code = ctypes.c_int(-1)
    _lib.check(_lib.load().ps_model_poll_status(b.handle, ctypes.byref(code)))
    assert code.value == 0


# ---------------------------------------------------------------------------
# trajectory cost + adjoint (workload 3) and rollouts (workload 4)
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def w3():
    wl = workloads.workload(3, scale=1.0 / 8)
    b, sc, om, ref = make(wl["asset"], wl["obbs"])
    return wl, b, sc, om, ref


def _params(wl, smooth=0.0):
    return api.CostParams(collision_cost_weight=wl["w"], world_collision_margin=wl["eps"],
                          self_collision_margin=wl["self_margin"], smoothness_weight=smooth,
                          delta_t=wl["delta_t"])


def test_waypoint_cost_vs_fp64_and_reference(w3):
    wl, b, sc, om, ref = w3
    q = wl["q"]
    B, T, D = q.shape
    wp, tc, _ = api.traj_cost(b, sc, torch.from_numpy(q).cuda(), _params(wl), want_grad=False)
    ours = wp.cpu().numpy().reshape(-1)
    c64 = om.state_cost(q.reshape(-1, D), wl["w"], wl["eps"], wl["self_margin"])
    rel = np.abs(ours - c64) / np.maximum(np.abs(c64), 1.0)
    print(f"waypoint cost: max rel err vs fp64 = {rel.max():.2e}, active = {(c64 > 0).mean():.2f}")
    assert rel.max() < COST_REL_TOL
    rsc, _, _ = ref.chomp(q.transpose(0, 2, 1), wl["w"], wl["eps"], wl["self_margin"], grad=False)
    rref = rsc[:, 0, :].reshape(-1)
    relr = np.abs(ours - rref) / np.maximum(np.abs(rref), 1.0)
    print(f"waypoint cost: max rel diff vs reference kernel = {relr.max():.2e}")
    assert relr.max() < 1e-3
    np.testing.assert_allclose(tc.cpu().numpy(), ours.reshape(B, T).sum(1), rtol=1e-5, atol=1e-4)


def test_gradient_vs_fp64_central_difference(w3):
    wl, b, sc, om, ref = w3
    q = wl["q"][:16]
    B, T, D = q.shape
    _, _, g = api.traj_cost(b, sc, torch.from_numpy(q).cuda(), _params(wl))
    ours = g.cpu().numpy().reshape(-1, D)
    flat = q.reshape(-1, D)
    fd = om.state_cost_fd_grad(flat, wl["w"], wl["eps"], wl["self_margin"], h=1e-6)
    kink = om.kink_distance(flat, wl["eps"], wl["self_margin"])
    assert_gradient_vs_fd(ours, fd, kink, "gradient")


def test_gradient_vs_reference_fd_kernel(w3):
    wl, b, sc, om, ref = w3
    q = wl["q"][:4]
    _, _, g = api.traj_cost(b, sc, torch.from_numpy(q).cuda(), _params(wl))
    _, rg, _ = ref.chomp(q.transpose(0, 2, 1), wl["w"], wl["eps"], wl["self_margin"], state=False)
    rg = rg.transpose(0, 2, 1)
    ours = g.cpu().numpy()
    ours[:, 0, :] = 0.0
    ours[:, -1, :] = 0.0     # the reference pins endpoints
    gap = np.linalg.norm(ours - rg) / max(np.linalg.norm(rg), 1e-12)
    print(f"gradient: rel L2 gap to the reference FD kernel (eps=1e-3) = {gap:.2e}")
    assert gap < 0.25


def test_smoothness_term_matches_dense_R(w3):
    wl, b, sc, om, ref = w3
    q = wl["q"][:8]
    B, T, D = q.shape
    _, tc0, g0 = api.traj_cost(b, sc, torch.from_numpy(q).cuda(), _params(wl, 0.0))
    _, tc1, g1 = api.traj_cost(b, sc, torch.from_numpy(q).cuda(), _params(wl, 1.0))
    R = oracle.control_cost_R(T, wl["delta_t"])
    qd = q.astype(np.float64)
    sm = np.einsum("btd,ts,bsd->b", qd, R, qd)
    gs = 2.0 * np.einsum("ts,bsd->btd", R, qd)
    np.testing.assert_allclose((tc1 - tc0).cpu().numpy(), sm, rtol=2e-4)
    np.testing.assert_allclose((g1 - g0).cpu().numpy(), gs, rtol=1e-3, atol=1e-2 * np.abs(gs).max())


def test_autograd_function(w3):
    """Forward is the cost kernel alone; backward recomputes FK and runs the
    adjoint kernel; the result is the fused call's gradient scaled by
    grad_output. Double backward is refused."""
    wl, b, sc, om, ref = w3
    q = torch.from_numpy(wl["q"][:4]).cuda().requires_grad_(True)
    cost = api.hinge_cost(q, b, sc, _params(wl, 0.5))
    _, tc, g = api.traj_cost(b, sc, q.detach(), _params(wl, 0.5))
    torch.testing.assert_close(cost.detach(), tc, rtol=1e-6, atol=1e-5)
    (cost * torch.arange(1, 5, device="cuda")).sum().backward()
    assert torch.equal(q.grad, g * torch.arange(1, 5, device="cuda", dtype=torch.float32).view(-1, 1, 1))
    q2 = torch.from_numpy(wl["q"][:2]).cuda().requires_grad_(True)
    (gq,) = torch.autograd.grad(api.hinge_cost(q2, b, sc, _params(wl, 0.5)).sum(), q2, create_graph=True)
    with pytest.raises(RuntimeError):
        gq.sum().backward()


def test_bdt_layout_equals_btd(w3):
    wl, b, sc, om, ref = w3
    q = torch.from_numpy(wl["q"][:4]).cuda()
    w1_, t1, g1 = api.traj_cost(b, sc, q, _params(wl, 1.0))
    w2_, t2, g2 = api.traj_cost(b, sc, q.transpose(1, 2).contiguous(), _params(wl, 1.0), layout=_lib.PS_LAYOUT_BDT)
    torch.testing.assert_close(w1_, w2_)
    torch.testing.assert_close(g1, g2.transpose(1, 2))


def test_rollout_costs_vs_reference_stomp():
    wl = workloads.workload(4, scale=1.0 / 32)
    b, sc, om, ref = make(wl["asset"], wl["obbs"])
    r = wl["rollouts"][:256]
    p = api.CostParams(collision_cost_weight=wl["w"], world_collision_margin=wl["eps"],
                       self_collision_margin=wl["self_margin"])
    ours = api.rollout_costs(b, sc, torch.from_numpy(r).cuda(), p, broadcast_d=True).cpu().numpy()
    theirs, _ = ref.stomp(r, wl["w"], wl["eps"], wl["self_margin"])
    rel = np.abs(ours - theirs) / np.maximum(np.abs(theirs), 1.0)
    print(f"rollout cost: max rel diff vs reference stomp kernel = {rel.max():.2e}")
    assert rel.max() < 1e-3
    R, D, T = r.shape
    c64 = om.state_cost(r.transpose(0, 2, 1).reshape(-1, D), wl["w"], wl["eps"], wl["self_margin"])
    rel64 = np.abs(ours[:, 0, :].reshape(-1) - c64) / np.maximum(np.abs(c64), 1.0)
    print(f"rollout cost: max rel err vs fp64 = {rel64.max():.2e}")
    assert rel64.max() < COST_REL_TOL


def test_rollout_costs_full_workload_vs_fp64():
    """All 409,600 rollout waypoints of workload 4 against the FP64 oracle.
    The self hinge culls against the smallest clearance found so far, so this
    covers the deep self overlaps (near-concentric spheres of two joints) that
    only some requests of the full workload reach, where a cull that rejected
    the minimum pair would lower the cost by several units."""
    wl = workloads.workload(4)
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    om = oracle.OracleModel(b, *wl["obbs"])
    r = wl["rollouts"]
    p = api.CostParams(collision_cost_weight=wl["w"], world_collision_margin=wl["eps"],
                       self_collision_margin=wl["self_margin"])
    ours = api.rollout_costs(b, sc, torch.from_numpy(r).cuda(), p).cpu().numpy().reshape(-1)
    R, D, T = r.shape
    q = r.transpose(0, 2, 1).reshape(-1, D)
    c64 = om.state_cost(q, wl["w"], wl["eps"], wl["self_margin"])
    no_self = om.state_cost(q, wl["w"], wl["eps"], -1.0e9)
    deep = int(((c64 - no_self) > wl["w"] * 0.1).sum())   # self term above w * 0.1: overlap deeper than 0.09 m
    rel = np.abs(ours - c64) / np.maximum(np.abs(c64), 1.0)
    print(f"rollout cost, full workload: max rel err vs fp64 = {rel.max():.2e}; "
          f"{deep} waypoints with a self overlap deeper than 0.09 m")
    assert deep > 0
    assert rel.max() < COST_REL_TOL


def test_edges_probe_path_bitexact():
    """The end-sample probe runs in front of the persistent queue when there
    are at least 8 edges per SM lane group (38 K on a B200): at 0.6 of
    workload 2 (39,321 edges) the persistent path, with the probe, equals the
    reference kernels and the probe-free plain path bit for bit."""
    wl = workloads.workload(2, scale=0.6)
    b, sc, om, ref = make(wl["asset"], wl["obbs"])
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    assert len(wl["G"]) >= 8 * 32 * n_sm
    f, t, g = (torch.from_numpy(x).cuda() for x in (wl["from"], wl["to"], wl["G"]))
    v, c, _ = api.check_edges(b, sc, f, t, samples=g)
    vp, cp, _ = api.check_edges(b, sc, f, t, samples=g, persistent=False)
    assert torch.equal(v, vp) and torch.equal(c.view(torch.int32), cp.view(torch.int32))
    rv, rc, _ = ref.check_edges(wl["from"], wl["to"], wl["G"])
    np.testing.assert_array_equal(v.cpu().numpy(), rv)
    assert np.array_equal(c.cpu().numpy().view(np.uint32), rc.view(np.uint32))
