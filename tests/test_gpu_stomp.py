"""Batched STOMP optimiser on the device (ps_stomp_optimize) against the
reference's iteration (STOMP::solve_runtime_scene, cpp/src/planning/
stomp.cu:565-965) restated on the host in FP64 with dense matrices.

* First iteration: the rollouts equal clamp(theta + L z) with the dense
  Cholesky factor L of stomp_precompute.cpp:46-68 and z from a NumPy
  restatement of the Philox4x32-10 + Box-Muller stream (within 2e-6 rad);
  state costs equal ps_rollout_costs' kernel bit for bit; row totals, the
  exponentiated weights, the weighted noise and the M projection
  (stomp.cu:257-413) give the updated optimum within 2e-5 rad.
* Second iteration: the reused rows are the reference's top-k selection of
  the previous row totals (stomp.cu:133-177), copied exactly.
* The bookkeeping equals the host restatement of stomp.cu:764-889 on
  independently computed totals and validity.
* Solved paths are collision-free under the FP64 oracle; a request's result
  does not depend on the batch it is solved in; the reference solver run on
  the same requests reports paths this library's check also accepts.
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import golden_asset
from prismplan_b200 import _lib, api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors
from stomp_host import normals, stomp_matrices
from test_gpu_chomp import _densify, _reference_bookkeeping

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(golden):
    """The reference's Panda, 16 random OBBs, 16 (start, goal) pairs with
    both endpoints collision-free (self check included)."""
    asset, _ = golden_asset(golden, "panda")
    rng = np.random.default_rng(1017)
    obbs = workloads.random_obbs(rng, 16)
    b = RobotModelBuilder.from_asset(asset).build()
    sc = SceneTensors(*obbs)

    def is_free(q):
        hit, _ = api.check_configs(b, sc, torch.from_numpy(q).cuda(), check_self=True)
        return hit.cpu().numpy() == 0

    starts, goals = workloads.free_pairs(rng, asset, 16, is_free)
    return asset, obbs, b, sc, starts, goals


def _settings(**kw):
    s = api.StompSettings(time_limit_ms=0.0)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _free_run(**kw):
    return _settings(num_iterations_after_valid=10 ** 6, convergence_eps=0.0, **kw)


def _ws_view(ws, offset, shape, dtype=np.float32):
    n = int(np.prod(shape)) * np.dtype(dtype).itemsize
    return ws[offset:offset + n].cpu().numpy().view(dtype).reshape(shape)


def _run(b, sc, theta0, s, ws=None):
    B, T, D = theta0.shape
    ws = ws if ws is not None else api.stomp_workspace(b, B, T, s)
    res = api.stomp_optimize(b, sc, torch.from_numpy(theta0).cuda(), s, workspace=ws)
    torch.cuda.synchronize()
    return res, ws


def _cost_params(s, smooth):
    return api.CostParams(collision_cost_weight=s.collision_cost_weight,
                          world_collision_margin=s.world_collision_margin,
                          self_collision_margin=s.self_collision_margin, include_self=s.include_self,
                          smoothness_weight=smooth, delta_t=s.delta_t)


def test_first_iteration_matches_host_restatement(case):
    asset, obbs, b, sc, starts, goals = case
    s = _free_run(num_iterations=1)
    T, B, D = s.num_timesteps, 4, b.n_dof
    Rn, Ro = s.num_rollouts_new, s.num_rollouts_old
    R = Rn + Ro + 1
    th0 = api.chomp_linear_init(b, starts[:B], goals[:B], T).cpu().numpy()
    res, ws = _run(b, sc, th0, s)
    lay = api.stomp_layout(b, B, T, s)
    roll = _ws_view(ws, lay["rollouts"][1], (R, B, T, D))
    noise = _ws_view(ws, lay["noise"], (R, B, T, D))
    scost = _ws_view(ws, lay["state_cost"][1], (R, B, T))
    rtot = _ws_view(ws, lay["row_total"][1], (R, B))
    lo = np.asarray(asset["joint_lower"], np.float32)
    hi = np.asarray(asset["joint_upper"], np.float32)
    Rm, L, M = stomp_matrices(T, s.delta_t, s.noise_scale)
    # rollouts: all Rn + Ro rows fresh on the first iteration, then the optimum
    z = normals(np.arange(Rn + Ro), D, T, 1, s.seed)                 # [rows, D, T]
    n = np.einsum("ts,rds->rdt", L, z)
    n[:, :, 0] = 0.0
    n[:, :, -1] = 0.0
    want = np.clip(th0[None] + n.transpose(0, 2, 1)[:, None].astype(np.float32), lo, hi)   # [rows, B, T, D]
    err = np.abs(roll[:Rn + Ro] - want).max()
    print(f"first iteration: max |rollout - clamp(theta + L z)| = {err:.2e}")
    assert err < 2e-6
    assert np.array_equal(roll[R - 1], th0) and not noise[R - 1].any()
    np.testing.assert_array_equal(noise, (roll - th0[None]).astype(np.float32))
    # state costs: the rollout-cost kernel's bits
    wp, _, _ = api.traj_cost(b, sc, torch.from_numpy(roll.reshape(R * B, T, D)).cuda(), _cost_params(s, 0.0),
                             want_grad=False)
    assert np.array_equal(scost.reshape(R * B, T).view(np.uint32), wp.cpu().numpy().view(np.uint32))
    # control costs and row totals (FP64, dense R)
    x = roll.astype(np.float64)                                        # [R, B, T, D]
    ctrl = s.control_cost_weight * x * np.einsum("ts,rbsd->rbtd", Rm, x)
    tot = scost.astype(np.float64).sum(2) + ctrl.sum((2, 3))
    np.testing.assert_allclose(rtot, tot, rtol=2e-5, atol=1e-4)
    # weights, weighted noise, projection (stomp.cu:314-413)
    c = scost.astype(np.float64)[..., None] + ctrl                      # [R, B, T, D]
    mn, mx = c.min(0), c.max(0)
    u = np.exp(-s.exponentiated_cost_sensitivity * (c - mn) / np.maximum(mx - mn, 1e-8))
    p = u / np.maximum(u.sum(0), 1e-12)
    delta = (p * noise.astype(np.float64)).sum(0)                       # [B, T, D]
    delta[:, 0] = 0.0
    delta[:, -1] = 0.0
    step = np.einsum("ts,bsd->btd", M, delta)
    step[:, 0] = 0.0
    step[:, -1] = 0.0
    th1 = th0 + step
    err = np.abs(res.theta.cpu().numpy() - th1).max()
    print(f"first iteration: max |theta_1 - FP64 restatement| = {err:.2e}, max |M delta| = {np.abs(step).max():.3f}")
    assert err < 2e-5


def test_second_iteration_reuses_top_k(case):
    asset, obbs, b, sc, starts, goals = case
    T, B, D = 51, 3, b.n_dof
    s1 = _free_run(num_iterations=1)
    Rn, Ro = s1.num_rollouts_new, s1.num_rollouts_old
    R = Rn + Ro + 1
    th0 = api.chomp_linear_init(b, starts[:B], goals[:B], T).cpu().numpy()
    r1, _ = _run(b, sc, th0, s1)
    s2 = _free_run(num_iterations=2)
    r2, ws = _run(b, sc, th0, s2)
    lay = api.stomp_layout(b, B, T, s2)
    roll1 = _ws_view(ws, lay["rollouts"][1], (R, B, T, D))
    tot1 = _ws_view(ws, lay["row_total"][1], (R, B))
    sc1 = _ws_view(ws, lay["state_cost"][1], (R, B, T))
    roll2 = _ws_view(ws, lay["rollouts"][0], (R, B, T, D))
    sc2 = _ws_view(ws, lay["state_cost"][0], (R, B, T))
    idx = _ws_view(ws, lay["reuse_index"], (B, Ro), np.int32)
    th1 = r1.theta.cpu().numpy()
    for i in range(B):
        cc = tot1[:, i].copy()
        want = []
        for _ in range(Ro):   # stomp_select_topk_kernel
            k = int(np.argmin(cc))
            want.append(k)
            cc[k] = np.float32(3.0e38)
        assert idx[i].tolist() == want, i
        np.testing.assert_array_equal(roll2[Rn:Rn + Ro, i], roll1[want, i])
        np.testing.assert_array_equal(sc2[Rn:Rn + Ro, i], sc1[want, i])
        np.testing.assert_array_equal(roll2[R - 1, i], th1[i])
    # fresh rows of iteration 2 draw step 2 of the stream, around theta_1
    Rm, L, M = stomp_matrices(T, 0.1, 1.0)
    z = normals(np.arange(Rn), D, T, 2, s2.seed)
    n = np.einsum("ts,rds->rdt", L, z)
    n[:, :, 0] = n[:, :, -1] = 0.0
    lo = np.asarray(asset["joint_lower"], np.float32)
    hi = np.asarray(asset["joint_upper"], np.float32)
    want = np.clip(th1[None] + n.transpose(0, 2, 1)[:, None].astype(np.float32), lo, hi)
    assert np.abs(roll2[:Rn] - want).max() < 2e-6


def test_bookkeeping_matches_reference_loop(case):
    asset, obbs, b, sc, starts, goals = case
    N, B, T = 8, 12, 51
    th0 = api.chomp_linear_init(b, starts[:B], goals[:B], T).cpu().numpy()
    base = _free_run()
    thetas = []
    for k in range(N + 1):
        base.num_iterations = k
        thetas.append(_run(b, sc, th0, base)[0].theta.cpu().numpy())
    s = _settings(num_iterations=N, num_iterations_after_valid=2, convergence_eps=1e-4)
    totals, valids = [], []
    for t in thetas:
        _, tc, _ = api.traj_cost(b, sc, torch.from_numpy(t).cuda(), _cost_params(s, s.control_cost_weight),
                                 want_grad=False)
        totals.append(tc.cpu().numpy())
        pts = [_densify(x, s.collision_check_step) for x in t]
        hit, _ = api.check_configs(b, sc, torch.from_numpy(np.concatenate(pts)).cuda(), check_self=True)
        hit = hit.cpu().numpy().astype(bool)
        o, v = 0, []
        for p in pts:
            v.append(not hit[o:o + len(p)].any())
            o += len(p)
        valids.append(v)
    totals, valids = np.stack(totals), np.array(valids)
    res, _ = _run(b, sc, th0, s)
    solved, iters = res.solved.cpu().numpy(), res.iterations.cpu().numpy()
    cost, path = res.cost.cpu().numpy(), res.path.cpu().numpy()
    print(f"valid per step: {valids.sum(1).tolist()}; solved {solved.sum()} of {B}; iterations {iters.tolist()}")
    assert valids.any() and not valids.all()
    for i in range(B):
        bv, it, bk, bt = _reference_bookkeeping(totals[:, i], valids[:, i], s)
        assert bool(solved[i]) == bv, i
        assert iters[i] == it, (i, iters[i], it)
        assert cost[i].view(np.uint32) == np.float32(bt).view(np.uint32), (i, cost[i], bt)
        assert np.array_equal(path[i], thetas[bk][i] if bv else thetas[it][i]), i


def test_solve_invariants_batch_independence_and_reference(case):
    asset, obbs, b, sc, starts, goals = case
    s = _settings()   # the reference's defaults: T = 51, 20 iterations, 30 + 20 rollouts
    res = api.stomp_solve(b, sc, starts, goals, s)
    path, solved = res.path.cpu().numpy(), res.solved.cpu().numpy()
    iters = res.iterations.cpu().numpy()
    B = len(starts)
    np.testing.assert_array_equal(path[:, 0], starts)
    np.testing.assert_array_equal(path[:, -1], goals)
    assert (iters >= 0).all() and (iters <= s.num_iterations).all()
    # a request's result does not depend on its batch
    for i in (0, 5, 11):
        one = api.stomp_solve(b, sc, starts[i:i + 1], goals[i:i + 1], s)
        assert np.array_equal(one.path.cpu().numpy()[0], path[i]), i
        assert one.iterations.cpu().numpy()[0] == iters[i]
    # solved paths are collision-free under the FP64 oracle (flips only at contact)
    om = oracle.OracleModel(b, *obbs)
    for i in np.nonzero(solved)[0]:
        pts = _densify(path[i], s.collision_check_step)
        hit, _, gap = om.check_configs(pts, margin=s.collision_margin, flags=_lib.PS_CHECK_SELF)
        assert not hit.any() or np.abs(gap[hit.astype(bool)]).max() < 1e-5, i
    ref = oracle.RefKernels(b, *obbs)
    rpath, rsolved, riters, _, ms = ref.stomp_solve(starts, goals, s.num_timesteps, s.to_c())
    print(f"solved: device {solved.sum()} of {B} (mean iterations {iters.mean():.1f}); reference "
          f"{rsolved.sum()} of {B} (mean iterations {riters.mean():.1f}, {ms / B:.2f} ms per request)")
    assert solved.sum() > B // 4 and rsolved.sum() > B // 4
    pts_ok = []
    for i in np.nonzero(rsolved)[0]:
        pts = _densify(rpath[i], s.collision_check_step)
        hit, _ = api.check_configs(b, sc, torch.from_numpy(pts).cuda(), check_self=True)
        pts_ok.append(not hit.cpu().numpy().any())
    assert all(pts_ok)


def test_edge_cases(case):
    asset, obbs, b, sc, starts, goals = case
    th0 = api.chomp_linear_init(b, starts[:3], goals[:3], 24).cpu().numpy()
    # no reuse rows, a single new rollout
    res, _ = _run(b, sc, th0, _settings(num_iterations=3, num_rollouts_old=0, num_rollouts_new=1))
    assert np.isfinite(res.theta.cpu().numpy()).all()
    # T = 2: nothing to move
    t2 = np.ascontiguousarray(th0[:, [0, -1]])
    res, _ = _run(b, sc, t2, _settings(num_iterations=2))
    assert np.array_equal(res.theta.cpu().numpy(), t2)
    # invalid sizes
    with pytest.raises(_lib.PrismError):
        api.stomp_optimize(b, sc, torch.zeros((1, 1025, b.n_dof), device="cuda"), _settings())
    with pytest.raises(ValueError):
        api.stomp_workspace(b, 1, 16, _settings(num_rollouts_new=0))
    ws = torch.empty(256, dtype=torch.uint8, device="cuda")
    with pytest.raises(_lib.PrismError):
        api.stomp_optimize(b, sc, torch.from_numpy(th0).cuda(), _settings(), workspace=ws)
