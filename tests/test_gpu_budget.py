"""Time budget of the persistent edge paths (failure detection without a GPU
fault): a budget that runs out stops the queue kernels, reports PS_ETIMEOUT
and never reports an unfinished edge as free; a generous budget changes
nothing; the next call starts clean."""
import numpy as np
import pytest
import torch

from prismplan_b200 import _lib, api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def w2():
    wl = workloads.workload(2, scale=1.0 / 16)
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    frm = torch.from_numpy(wl["from"]).cuda()
    to = torch.from_numpy(wl["to"]).cuda()
    return b, sc, frm, to


def _params(budget):
    return api.EdgeEvalParams(max_joint_step=0.01, max_samples=600, time_budget_ms=budget)


@pytest.mark.parametrize("static", [False, True])
def test_budget_runs_out_without_false_free(w2, static):
    b, sc, frm, to = w2
    ws = None if static else api.edges_workspace(len(frm))
    run = (lambda p: _static(b, sc, frm, to, p)) if static else (
        lambda p: api.check_edges(b, sc, frm, to, params=p, workspace=ws))
    v_ref, c_ref, _ = run(_params(0.0))
    torch.cuda.synchronize()
    assert api.edges_status(ws) == _lib.PS_OK
    v_to, c_to, _ = run(_params(1.0e-6))   # about 1 ns: every queue kernel stops at its first grab
    torch.cuda.synchronize()
    assert api.edges_status(ws) == _lib.PS_ETIMEOUT
    v_ref, v_to = v_ref.cpu().numpy(), v_to.cpu().numpy()
    assert not np.any((v_to == 1) & (v_ref == 0))          # never free when not shown free
    assert (v_to == 0).mean() > (v_ref == 0).mean()          # unfinished edges came back invalid
    assert np.all(c_to.cpu().numpy()[v_to == 0] == np.finfo(np.float32).max)
    # a generous budget changes nothing, and the status resets
    v_ok, c_ok, _ = run(_params(10000.0))
    torch.cuda.synchronize()
    assert api.edges_status(ws) == _lib.PS_OK
    np.testing.assert_array_equal(v_ok.cpu().numpy(), v_ref)
    assert torch.equal(c_ok.cpu().view(torch.int32), c_ref.cpu().view(torch.int32))


def _static(b, sc, frm, to, p):
    import ctypes as C

    E = frm.shape[0]
    v = torch.empty(E, dtype=torch.uint8, device="cuda")
    c = torch.empty(E, dtype=torch.float32, device="cuda")
    k = torch.empty(E, dtype=torch.float32, device="cuda")
    pc = p.to_c()
    view = sc.view()
    _lib.check(_lib.load().ps_check_edges_static(b.handle, C.byref(view), frm.data_ptr(), to.data_ptr(), None, E,
                                                 C.byref(pc), v.data_ptr(), c.data_ptr(), k.data_ptr(), None))
    return v, c, k


def test_batch_budget(w2):
    b, sc, frm, to = w2
    E = frm.shape[0]
    batch = api.MixedBatch(b, 4, E, 0, 0, 0)
    outs = [batch.add_edges(frm[i::4], to[i::4]) for i in range(4)]
    batch.launch(sc, _params(1.0e-6), api.CostParams())
    assert batch.status() == _lib.PS_ETIMEOUT
    v_to = torch.cat([o[0] for o in outs]).cpu().numpy()
    batch.launch(sc, _params(0.0), api.CostParams())
    assert batch.status() == _lib.PS_OK
    v_ref = torch.cat([o[0] for o in outs]).cpu().numpy()
    assert not np.any((v_to == 1) & (v_ref == 0))
    assert v_ref.mean() > 0.0
    batch.close()
