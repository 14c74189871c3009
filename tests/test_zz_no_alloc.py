"""GPU: edge checks through ps_check_edges_static, the entry point for callers
that cannot allocate device memory (a planner inside a per-expansion latency
budget, a host process without its own CUDA allocator). Its workspace is a
device array built into the library; the test checks that two calls in a row
give exactly the verdicts and costs of ps_check_edges with a caller-provided
workspace, and that oversized batches are refused.

Kept in a file of its own, collected last, and self-contained: it must pass
in a fresh process as well as after every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from prismplan_b200 import _lib, api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu


def _call_static(lib, b, view, frm, to, G, params, out):
    valid, cost, clr = out
    return lib.ps_check_edges_static(b.handle, C.byref(view), frm.data_ptr(), to.data_ptr(),
                                     G.data_ptr() if G is not None else None, frm.shape[0], C.byref(params),
                                     valid.data_ptr(), cost.data_ptr(), clr.data_ptr(), None)


@pytest.mark.parametrize("use_given_samples", [True, False])
def test_static_workspace_matches_caller_workspace(use_given_samples):
    wl = workloads.workload(2, scale=1.0 / 16)          # 4096 edges, uneven 1..600 samples
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    frm = torch.from_numpy(wl["from"]).cuda()
    to = torch.from_numpy(wl["to"]).cuda()
    G = torch.from_numpy(wl["G"]).cuda() if use_given_samples else None
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    v_ref, c_ref, _ = api.check_edges(b, sc, frm, to, samples=G, params=p)   # caller-provided workspace
    torch.cuda.synchronize()
    lib = _lib.load()
    view = sc.view()
    cp = p.to_c()
    E = frm.shape[0]
    for call in range(2):   # the second call reuses the array the first one left behind
        out = (torch.full((E,), 7, dtype=torch.uint8, device="cuda"), torch.full((E,), -1.0, device="cuda"),
               torch.full((E,), -1.0, device="cuda"))
        _lib.check(_call_static(lib, b, view, frm, to, G, cp, out))
        torch.cuda.synchronize()
        assert torch.equal(out[0], v_ref), f"call {call}: verdicts differ"
        assert np.array_equal(out[1].cpu().numpy().view(np.uint32), c_ref.cpu().numpy().view(np.uint32)), \
            f"call {call}: costs differ"
    assert 0.02 < float(v_ref.float().mean()) < 0.98


def test_static_workspace_at_full_capacity():
    """65,536 edges, the array's limit: the per-edge segments fill it exactly
    and the end-sample probe runs in front of the queue (it starts at 8 warps
    of edges per SM), as on the persistent path."""
    wl = workloads.workload(2)                          # 65,536 edges, 1..600 samples each
    E = len(wl["from"])
    assert E == _lib.PS_EDGES_STATIC_MAX
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    frm = torch.from_numpy(wl["from"]).cuda()
    to = torch.from_numpy(wl["to"]).cuda()
    G = torch.from_numpy(wl["G"]).cuda()
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    v_ref, c_ref, _ = api.check_edges(b, sc, frm, to, samples=G, params=p)
    torch.cuda.synchronize()
    lib = _lib.load()
    view, cp = sc.view(), p.to_c()
    for call in range(2):
        out = (torch.full((E,), 7, dtype=torch.uint8, device="cuda"), torch.full((E,), -1.0, device="cuda"),
               torch.full((E,), -1.0, device="cuda"))
        _lib.check(_call_static(lib, b, view, frm, to, G, cp, out))
        torch.cuda.synchronize()
        assert torch.equal(out[0], v_ref), f"call {call}: verdicts differ"
        assert np.array_equal(out[1].cpu().numpy().view(np.uint32), c_ref.cpu().numpy().view(np.uint32))
    st = C.c_int(-1)
    _lib.check(lib.ps_edges_status(None, C.byref(st)))
    assert st.value == _lib.PS_OK


def test_static_workspace_rejects_oversized_batch():
    wl = workloads.workload(2, scale=1.0 / 16)
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    E = 65536 + 1
    frm = torch.zeros((E, 7), device="cuda")
    out = (torch.empty(E, dtype=torch.uint8, device="cuda"), torch.empty(E, device="cuda"),
           torch.empty(E, device="cuda"))
    lib = _lib.load()
    rc = _call_static(lib, b, sc.view(), frm, frm, None, api.EdgeEvalParams(granularity=4).to_c(), out)
    assert rc == _lib.PS_EINVAL
    assert b"exceeds the built-in workspace" in lib.ps_last_error()
