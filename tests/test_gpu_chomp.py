"""Batched CHOMP optimiser on the device (ps_chomp_optimize) against the
reference's iteration (CHOMP::solve_runtime_scene, cpp/src/planning/
chomp.cu:358-600) restated on the host.

* One update equals the FP64 covariant step of chomp_update_kernel
  (chomp.cu:259-289) on the same obstacle gradient: within 2e-6 rad.
* The device bookkeeping (best valid snapshot, polish budget, convergence
  streak, iteration count) equals a host restatement of chomp.cu:487-537
  driven by independently computed costs and validity (ps_traj_cost,
  ps_check_configs over the densified points of chomp.cu:320-333): exact.
* Solved paths are collision-free under the FP64 oracle (flips only at
  contact), pinned at start and goal, inside the limits; best_cost equals the
  recomputed total cost bit for bit.
* The reference solver itself (oracle/_ref) on the same requests: every path
  it reports solved is valid under this library's check as well.
"""
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
def w3():
    wl = workloads.workload(3, scale=1.0 / 8)   # 32 trajectories, T = 64, Panda-like, 64 OBBs
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    return wl, b, sc


@pytest.fixture(scope="module")
def solve_case(golden):
    """The reference's Panda asset, 16 random OBBs, 24 (start, goal) pairs
    with both endpoints collision-free (self check included)."""
    asset, _ = golden_asset(golden, "panda")
    rng = np.random.default_rng(1017)   # a field that leaves about 70 % of configurations free
    obbs = workloads.random_obbs(rng, 16)
    b = RobotModelBuilder.from_asset(asset).build()
    sc = SceneTensors(*obbs)

    def is_free(q):
        hit, _ = api.check_configs(b, sc, torch.from_numpy(q).cuda(), check_self=True)
        return hit.cpu().numpy() == 0

    starts, goals = workloads.free_pairs(rng, asset, 24, is_free)
    wl = {"asset": asset, "obbs": obbs, "w": 20.0, "eps": 0.02, "self_margin": 0.01, "delta_t": 0.1}
    return wl, b, sc, starts, goals


def _settings(wl, **kw):
    s = api.ChompSettings(collision_cost_weight=wl["w"], world_collision_margin=wl["eps"],
                          self_collision_margin=wl["self_margin"], delta_t=wl["delta_t"], time_limit_ms=0.0)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _free_run(wl, **kw):
    """Settings under which no trajectory finishes before num_iterations."""
    return _settings(wl, num_iterations_after_valid=10 ** 6, convergence_eps=0.0, **kw)


def _cost_params(s: api.ChompSettings, smooth: float):
    return api.CostParams(collision_cost_weight=s.collision_cost_weight,
                          world_collision_margin=s.world_collision_margin,
                          self_collision_margin=s.self_collision_margin, include_self=s.include_self,
                          smoothness_weight=smooth, delta_t=s.delta_t)


def _densify(theta, step):
    """Points of chomp_validity_kernel (chomp.cu:320-333) for one trajectory:
    a + (b - a) * (s / n_sub), s = 0..n_sub-1 per segment, then the last
    waypoint; n_sub from the FP32 max segment length (chomp.cu:462-474)."""
    th = theta.astype(np.float32)
    T = len(th)
    diff = th[1:] - th[:-1]
    d2 = np.zeros(T - 1, np.float32)
    for d in range(th.shape[1]):   # in order, FP32, as the host loop
        d2 = (d2 + diff[:, d] * diff[:, d]).astype(np.float32)
    seg = np.sqrt(d2).astype(np.float32)
    mx = np.float32(seg.max()) if T > 1 else np.float32(0)
    n_sub = 1
    if step > 0 and mx > np.float32(step):
        n_sub = int(np.ceil(np.float32(mx) / np.float32(step)))
    frac = (np.arange(n_sub, dtype=np.float32) / np.float32(n_sub)).astype(np.float32)
    a = th[:-1, None, :].astype(np.float64)
    d = diff[:, None, :].astype(np.float64)
    pts = (d * frac[None, :, None].astype(np.float64) + a).astype(np.float32)   # one fused multiply-add
    return np.concatenate([pts.reshape(-1, th.shape[1]), th[-1:]], 0)


def _valid(b, sc, theta_b, s: api.ChompSettings):
    pts = [_densify(t, s.collision_check_step) for t in theta_b]
    q = torch.from_numpy(np.concatenate(pts, 0)).cuda()
    hit, _ = api.check_configs(b, sc, q, collision_margin=s.collision_margin, check_self=s.check_self)
    hit = hit.cpu().numpy().astype(bool)
    out, o = [], 0
    for p in pts:
        out.append(not hit[o:o + len(p)].any())
        o += len(p)
    return np.array(out)


def _total(b, sc, theta_b, s):
    wp, tc, _ = api.traj_cost(b, sc, torch.from_numpy(theta_b).cuda(), _cost_params(s, s.smoothness_weight))
    return tc.cpu().numpy()


def test_one_update_matches_fp64_step(w3):
    wl, b, sc = w3
    s = _free_run(wl, num_iterations=1)
    th0 = wl["q"][:8].copy()
    B, T, D = th0.shape
    res = api.chomp_optimize(b, sc, torch.from_numpy(th0).cuda(), s)
    got = res.theta.cpu().numpy()
    _, _, g = api.traj_cost(b, sc, torch.from_numpy(th0).cuda(), _cost_params(s, 0.0))
    og = g.cpu().numpy().astype(np.float64)
    og[:, 0, :] = 0.0
    og[:, -1, :] = 0.0
    R = workloads.control_cost_R(T, s.delta_t)
    A = R + 1e-8 * np.eye(T)
    th64 = th0.astype(np.float64)
    rhs = og + s.smoothness_weight * np.einsum("ts,bsd->btd", R, th64)
    x = np.linalg.solve(A[None], rhs)
    want = th64 - np.float64(np.float32(s.step_size)) * x
    lo = np.asarray(wl["asset"]["joint_lower"], np.float32)
    hi = np.asarray(wl["asset"]["joint_upper"], np.float32)
    want = np.clip(want.astype(np.float32), lo, hi)
    want[:, 0, :] = th0[:, 0, :]
    want[:, -1, :] = th0[:, -1, :]
    err = np.abs(got - want).max()
    print(f"one CHOMP update: max |theta - FP64 step| = {err:.2e} rad, max |step x| = "
          f"{np.abs(s.step_size * x).max():.3f}")
    assert err < 2e-6
    assert np.array_equal(got[:, 0], th0[:, 0]) and np.array_equal(got[:, -1], th0[:, -1])


def _reference_bookkeeping(totals, valids, s):
    """chomp.cu:487-537 on per-step totals / validity (step 0 = the seed)."""
    best_total, best_k, best_valid = np.inf, -1, False
    if valids[0]:
        best_total, best_k, best_valid = totals[0], 0, True
    polish, prev, streak, iters = s.num_iterations_after_valid, np.inf, 0, 0
    for it in range(s.num_iterations):
        if best_valid and polish <= 0:
            break
        k = it + 1
        iters += 1
        if valids[k] and totals[k] < best_total:
            best_total, best_k, best_valid = totals[k], k, True
        if best_valid:
            impr = np.float32(prev) - np.float32(best_total)
            streak = streak + 1 if (impr >= 0 and impr < np.float32(s.convergence_eps)) else 0
            prev = best_total
            polish -= 1
            if streak >= 2:
                break
    return best_valid, iters, best_k, (best_total if best_valid else totals[iters])


def test_bookkeeping_matches_reference_loop(solve_case):
    wl, b, sc, starts, goals = solve_case
    N = 12
    th0 = api.chomp_linear_init(b, starts[:12], goals[:12], 51).cpu().numpy()
    B = len(th0)
    base = _free_run(wl)
    thetas = []
    for k in range(N + 1):
        base.num_iterations = k
        thetas.append(api.chomp_optimize(b, sc, torch.from_numpy(th0).cuda(), base).theta.cpu().numpy())
    s = _settings(wl, num_iterations=N, num_iterations_after_valid=3, convergence_eps=1e-4)
    totals = np.stack([_total(b, sc, t, s) for t in thetas])        # [N+1, B]
    valids = np.stack([_valid(b, sc, t, s) for t in thetas])        # [N+1, B]
    res = api.chomp_optimize(b, sc, torch.from_numpy(th0).cuda(), s)
    solved = res.solved.cpu().numpy()
    iters = res.iterations.cpu().numpy()
    cost = res.cost.cpu().numpy()
    path = res.path.cpu().numpy()
    print(f"valid per step: {valids.sum(1).tolist()}; solved {solved.sum()} of {B}; iterations {iters.tolist()}")
    assert valids.any() and not valids.all()    # both branches of the bookkeeping are exercised
    for i in range(B):
        bv, it, bk, bt = _reference_bookkeeping(totals[:, i], valids[:, i], s)
        assert bool(solved[i]) == bv, i
        assert iters[i] == it, (i, iters[i], it)
        assert cost[i].view(np.uint32) == np.float32(bt).view(np.uint32), (i, cost[i], bt)
        want = thetas[bk][i] if bv else thetas[it][i]
        assert np.array_equal(path[i], want), i


def test_solve_invariants_and_reference_solver(solve_case):
    wl, b, sc, starts, goals = solve_case
    s = _settings(wl)   # the reference's defaults: T = 51, 100 iterations, 5 after valid
    res = api.chomp_solve(b, sc, starts, goals, s)
    path = res.path.cpu().numpy()
    solved = res.solved.cpu().numpy()
    iters = res.iterations.cpu().numpy()
    B, T, D = path.shape
    assert T == s.num_timesteps
    np.testing.assert_array_equal(path[:, 0], starts)
    np.testing.assert_array_equal(path[:, -1], goals)
    lo = np.asarray(wl["asset"]["joint_lower"], np.float32)
    hi = np.asarray(wl["asset"]["joint_upper"], np.float32)
    assert (path >= lo).all() and (path <= hi).all()
    assert (iters >= 0).all() and (iters <= s.num_iterations).all()
    # best_cost is the total cost of the returned path, bit for bit
    tot = _total(b, sc, path, s)
    assert np.array_equal(tot.view(np.uint32), res.cost.cpu().numpy().view(np.uint32))
    # solved paths are collision-free under the FP64 oracle (flips only at contact)
    om = oracle.OracleModel(b, *wl["obbs"])
    for i in np.nonzero(solved)[0]:
        pts = _densify(path[i], s.collision_check_step)
        hit, _, gap = om.check_configs(pts, margin=s.collision_margin, flags=_lib.PS_CHECK_SELF)
        assert not hit.any() or np.abs(gap[hit.astype(bool)]).max() < 1e-5, i
    # the reference solver on the same requests (one request at a time)
    ref = oracle.RefKernels(b, *wl["obbs"])
    rpath, rsolved, riters, rtotal, ms = ref.chomp_solve(starts, goals, s.num_timesteps, s.to_c())
    print(f"solved: device {solved.sum()} of {B} (mean iterations {iters.mean():.1f}); reference "
          f"{rsolved.sum()} of {B} (mean iterations {riters.mean():.1f}, {ms / B:.2f} ms per request)")
    assert solved.sum() > B // 4 and rsolved.sum() > B // 4
    if rsolved.any():
        assert _valid(b, sc, rpath[rsolved.astype(bool)], s).all()


def test_time_limit_and_edge_cases(solve_case):
    wl, b, sc, starts, goals = solve_case
    th0 = api.chomp_linear_init(b, starts[:6], goals[:6], 40).cpu().numpy()
    # a time limit that has passed by the first bookkeeping: the seed is final
    s = _settings(wl, time_limit_ms=1e-6)
    res = api.chomp_optimize(b, sc, torch.from_numpy(th0).cuda(), s)
    assert (res.iterations.cpu().numpy() == 0).all()
    assert np.array_equal(res.theta.cpu().numpy(), th0)
    v0 = _valid(b, sc, th0, s)
    assert np.array_equal(res.solved.cpu().numpy(), v0)
    # num_iterations = 0: evaluate only
    res = api.chomp_optimize(b, sc, torch.from_numpy(th0).cuda(), _settings(wl, num_iterations=0))
    assert (res.iterations.cpu().numpy() == 0).all()
    # T = 2: nothing to move
    t2 = np.ascontiguousarray(th0[:, [0, -1]])
    res = api.chomp_optimize(b, sc, torch.from_numpy(t2).cuda(), _settings(wl, num_iterations=3))
    assert np.array_equal(res.theta.cpu().numpy(), t2)
    # B = 0, T out of range, workspace too small
    lib = _lib.load()
    p = _settings(wl).to_c()
    v = sc.view()
    assert lib.ps_chomp_optimize(b.handle, C.byref(v), None, 0, 16, C.byref(p), None, None, None, None, None, 0,
                                 None) == _lib.PS_OK
    with pytest.raises(_lib.PrismError):
        api.chomp_optimize(b, sc, torch.zeros((1, 1025, b.n_dof), device="cuda"), _settings(wl))
    with pytest.raises(_lib.PrismError):
        api.chomp_optimize(b, sc, torch.zeros((1, 1, b.n_dof), device="cuda"), _settings(wl))
    ws = torch.empty(256, dtype=torch.uint8, device="cuda")
    with pytest.raises(_lib.PrismError):
        api.chomp_optimize(b, sc, torch.from_numpy(th0).cuda(), _settings(wl), workspace=ws)


def test_update_joint_limits_equals_rebuild(solve_case):
    """update_joint_limits (bindings.cpp:181-205) reaches the device: CHOMP
    clamps its updates to the model's limits (chomp.cu:259-289), and a model
    whose limits were narrowed in place gives the same bits as one built with
    the narrowed limits, inside those limits."""
    wl, _, sc, starts, goals = solve_case
    asset = wl["asset"]
    lo = np.asarray(asset["joint_lower"], np.float32)
    hi = np.asarray(asset["joint_upper"], np.float32)
    mid, half = (lo + hi) * 0.5, (hi - lo) * 0.25
    lo2, hi2 = (mid - half).astype(np.float32), (mid + half).astype(np.float32)
    st, gl = np.clip(starts[:8], lo2, hi2), np.clip(goals[:8], lo2, hi2)
    s = _free_run(wl, num_iterations=40)
    moved = RobotModelBuilder.from_asset(asset).build()
    wide = api.chomp_solve(moved, sc, st, gl, s).path.cpu().numpy()
    moved.joint_lower, moved.joint_upper = lo2.tolist(), hi2.tolist()
    moved.update_joint_limits()
    fresh = RobotModelBuilder.from_asset(dict(asset, joint_lower=lo2.tolist(), joint_upper=hi2.tolist())).build()
    a = api.chomp_solve(moved, sc, st, gl, s).path.cpu().numpy()
    f = api.chomp_solve(fresh, sc, st, gl, s).path.cpu().numpy()
    outside = ((wide < lo2) | (wide > hi2)).mean()
    print(f"share of waypoint values outside the narrowed limits with the original ones: {outside:.3f}")
    assert np.array_equal(a.view(np.uint32), f.view(np.uint32))
    assert (a >= lo2).all() and (a <= hi2).all()
    assert outside > 0
