"""GPU: the native host-buffer edge bridge (ps_edge_bridge_*, behind
api.EdgeEvalGpu), the counterpart of EdgeEvalGpu (edge_batch_bridge.hh:27-111).

Host arrays in, host arrays out. Its outputs must equal the device-resident
persistent path bit for bit (which the parity tests hold to the reference's
evaluate_edges_batch), and a slice of them the reference kernels directly:
over several staging slices and host threads, with graph replays fed
different edges, with clearance and the self check, under a time budget that
runs out, after a scene change, and for the argument errors the reference
raises on.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from prismplan_b200 import _lib, api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def w2():
    wl = workloads.workload(2, scale=0.75)   # 49,152 edges
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"])
    return wl, b, sc


def _device(b, sc, frm, to, p):
    v, c, k = api.check_edges(b, sc, torch.from_numpy(frm).cuda(), torch.from_numpy(to).cuda(), params=p)
    return v.cpu().numpy(), c.cpu().numpy(), k.cpu().numpy()


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def test_bridge_equals_device_path_and_reference(w2):
    wl, b, sc = w2
    E = len(wl["from"])
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    ev = api.EdgeEvalGpu(7, E, sc, b)
    rng = np.random.default_rng(7)
    for it in range(4):   # the first call runs eagerly, later ones replay the graph on new edges
        perm = rng.permutation(E)
        frm = np.ascontiguousarray(wl["from"][perm])
        to = np.ascontiguousarray(wl["to"][perm])
        v, c, k = ev.evaluate(frm.reshape(-1), to.reshape(-1), E, p)
        assert k.size == 0
        dv, dc, _ = _device(b, sc, frm, to, p)
        np.testing.assert_array_equal(v, dv)
        assert np.array_equal(_bits(c), _bits(dc))
    ref = oracle.RefKernels(b, *wl["obbs"])
    G = workloads.linf_samples(frm[:3000], to[:3000], 0.01)
    rv, rc, _ = ref.check_edges(frm[:3000], to[:3000], G)
    np.testing.assert_array_equal(v[:3000], rv)
    assert np.array_equal(_bits(c[:3000]), _bits(rc))
    assert ev.status() == _lib.PS_OK
    # fewer edges than the capacity, an odd count
    n = 9001
    v, c, _ = ev.evaluate(frm.reshape(-1), to.reshape(-1), n, p)
    dv, dc, _ = _device(b, sc, frm[:n], to[:n], p)
    np.testing.assert_array_equal(v, dv)
    assert np.array_equal(_bits(c), _bits(dc))
    # host arrays that are not the bridge's mirrors: the library stages them
    # itself, slice by slice (16,384 edges a slice; here 2 full slices, then
    # 3 slices with a partial last one)
    lib = _lib.load()
    pc = p.to_c()
    for n in (E, 40001 if E > 40001 else E - 1):
        perm = rng.permutation(E)[:n]
        f = np.ascontiguousarray(wl["from"][perm])
        t = np.ascontiguousarray(wl["to"][perm])
        v = np.empty(n, np.uint8)
        c = np.empty(n, np.float32)
        _lib.check(lib.ps_edge_bridge_evaluate(ev._h, f.ctypes.data, t.ctypes.data, n, C.byref(pc), v.ctypes.data,
                                               c.ctypes.data, None))
        dv, dc, _ = _device(b, sc, f, t, p)
        np.testing.assert_array_equal(v, dv)
        assert np.array_equal(_bits(c), _bits(dc))
    # edges written straight into the bridge's pinned input mirrors: no
    # staging copy (one copy in at full capacity, two below it)
    pf, pt = C.c_void_p(), C.c_void_p()
    _lib.check(lib.ps_edge_bridge_host_inputs(ev._h, C.byref(pf), C.byref(pt)))
    mf = np.ctypeslib.as_array(C.cast(pf, C.POINTER(C.c_float)), shape=(E, 7))
    mt = np.ctypeslib.as_array(C.cast(pt, C.POINTER(C.c_float)), shape=(E, 7))
    for n in (E, 12345):
        perm = rng.permutation(E)[:n]
        mf[:n] = wl["from"][perm]
        mt[:n] = wl["to"][perm]
        v = np.empty(n, np.uint8)
        c = np.empty(n, np.float32)
        _lib.check(lib.ps_edge_bridge_evaluate(ev._h, pf, pt, n, C.byref(pc), v.ctypes.data, c.ctypes.data, None))
        dv, dc, _ = _device(b, sc, np.ascontiguousarray(wl["from"][perm]), np.ascontiguousarray(wl["to"][perm]), p)
        np.testing.assert_array_equal(v, dv)
        assert np.array_equal(_bits(c), _bits(dc))
    del mf, mt
    ev.close()


def test_bridge_clearance_and_self_check():
    wl = workloads.workload(5, scale=0.5)
    b = RobotModelBuilder.from_asset(wl["asset"]).build()
    sc = SceneTensors(*wl["obbs"], *wl["esdf"])
    frm, to = wl["from"], wl["to"]
    E = len(frm)
    ev = api.EdgeEvalGpu(b.n_dof, E, sc, b)
    for p in (api.EdgeEvalParams(max_joint_step=0.01, max_samples=600, compute_clearance=True),
              api.EdgeEvalParams(max_joint_step=0.01, max_samples=600, check_self=True),
              api.EdgeEvalParams(granularity=24, check_self=True, compute_clearance=True, collision_margin=0.01)):
        for _ in range(2):
            v, c, k = ev.evaluate(frm.reshape(-1), to.reshape(-1), E, p)
            dv, dc, dk = _device(b, sc, frm, to, p)
            np.testing.assert_array_equal(v, dv)
            assert np.array_equal(_bits(c), _bits(dc))
            if p.compute_clearance:
                assert np.array_equal(_bits(k), _bits(dk))
            else:
                assert k.size == 0
        if not p.check_self:   # (this two-arm robot self-collides on every edge)
            assert 0.0 < v.mean() < 1.0
    ev.close()


def test_bridge_time_budget(w2):
    wl, b, sc = w2
    E = 4096
    frm, to = wl["from"][:E], wl["to"][:E]
    ev = api.EdgeEvalGpu(7, E, sc, b)
    ok = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    v_ref, c_ref, _ = ev.evaluate(frm, to, E, ok)
    assert ev.status() == _lib.PS_OK
    short = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600, time_budget_ms=1.0e-6)
    for _ in range(2):
        v, c, _ = ev.evaluate(frm, to, E, short)
        assert ev.status() == _lib.PS_ETIMEOUT
        assert not np.any((v == 1) & (v_ref == 0))
        assert np.all(c[v == 0] == np.finfo(np.float32).max)
    v2, c2, _ = ev.evaluate(frm, to, E, ok)
    assert ev.status() == _lib.PS_OK
    np.testing.assert_array_equal(v2, v_ref)
    assert np.array_equal(_bits(c2), _bits(c_ref))
    ev.close()


def test_bridge_scene_change(w2):
    wl, b, sc = w2
    E = 2048
    frm, to = wl["from"][:E], wl["to"][:E]
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    ev = api.EdgeEvalGpu(7, E, sc, b)
    v, _, _ = ev.evaluate(frm, to, E, p)
    assert v.mean() < 0.5
    empty = SceneTensors(np.zeros((0, 3), np.float32), np.zeros((0, 7), np.float32), np.zeros(0, np.uint8))
    ev.set_scene(empty)
    v0, c0, _ = ev.evaluate(frm, to, E, p)
    assert np.all(v0 == 1)
    np.testing.assert_allclose(c0, np.linalg.norm(to - frm, axis=1), rtol=1e-6)
    ev.set_scene(sc)
    v1, _, _ = ev.evaluate(frm, to, E, p)
    np.testing.assert_array_equal(v1, v)
    ev.close()


def test_bridge_argument_errors(w2):
    wl, b, sc = w2
    with pytest.raises(ValueError):
        api.EdgeEvalGpu(6, 16, sc, b)
    lib = _lib.load()
    h = C.c_void_p()
    view = sc.view()
    assert lib.ps_edge_bridge_create(b.handle, C.byref(view), 6, 16, C.byref(h)) == _lib.PS_EINVAL
    assert lib.ps_edge_bridge_create(b.handle, C.byref(view), 7, 0, C.byref(h)) == _lib.PS_EINVAL
    ev = api.EdgeEvalGpu(7, 16, sc, b)
    p = api.EdgeEvalParams(granularity=8)
    with pytest.raises(RuntimeError):
        ev.evaluate(wl["from"][:17], wl["to"][:17], 17, p)
    v, c, k = ev.evaluate(wl["from"][:0], wl["to"][:0], 0, p)
    assert v.size == 0 and c.size == 0 and k.size == 0
    with pytest.raises(ValueError):
        ev.evaluate(wl["from"][:3], wl["to"][:3], 4, p)
    pc = p.to_c()
    out = np.empty(16, np.uint8)
    cost = np.empty(16, np.float32)
    f = np.ascontiguousarray(wl["from"][:16])
    t = np.ascontiguousarray(wl["to"][:16])
    pc.compute_clearance = 1   # clearance asked for with no output array
    assert lib.ps_edge_bridge_evaluate(ev._h, f.ctypes.data, t.ctypes.data, 16, C.byref(pc), out.ctypes.data,
                                       cost.ctypes.data, None) == _lib.PS_EINVAL
    ev.close()
    ev.close()   # a second close is a no-op


def test_bridge_submit_wait_slots(w2):
    """Two slots in flight: every batch equals the synchronous call bit for bit,
    in a pipelined loop that submits one slot while the other runs."""
    wl, b, sc = w2
    E = 8192
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    ev = api.EdgeEvalGpu(7, E, sc, b)
    rng = np.random.default_rng(11)
    batches = []
    for k in range(6):
        n = E if k % 3 else 5000
        sel = rng.permutation(len(wl["from"]))[:n]
        batches.append((np.ascontiguousarray(wl["from"][sel]), np.ascontiguousarray(wl["to"][sel]), n))
    ref = [ev.evaluate(f, t, n, p) for f, t, n in batches]
    outs = [None] * len(batches)
    ev.submit(*batches[0], p, slot=0)
    for k in range(1, len(batches) + 1):
        if k < len(batches):
            ev.submit(*batches[k], p, slot=k % 2)
        outs[k - 1] = ev.wait((k - 1) % 2)
    for (v, c, _), (rv, rc, _) in zip(outs, ref):
        np.testing.assert_array_equal(v, rv)
        assert np.array_equal(_bits(c), _bits(rc))
    assert ev.status() == _lib.PS_OK
    # one call per slot at a time; waiting needs a call
    ev.submit(*batches[0], p, slot=1)
    with pytest.raises(RuntimeError):
        ev.submit(*batches[1], p, slot=1)
    lib = _lib.load()
    pc = p.to_c()
    f, t, n = batches[1]
    assert lib.ps_edge_bridge_submit(ev._h, 1, f.ctypes.data, t.ctypes.data, n, C.byref(pc)) == _lib.PS_EINVAL
    assert lib.ps_edge_bridge_submit(ev._h, 2, f.ctypes.data, t.ctypes.data, n, C.byref(pc)) == _lib.PS_EINVAL
    v, c, _ = ev.wait(1)
    np.testing.assert_array_equal(v, ref[0][0])
    with pytest.raises(RuntimeError):
        ev.wait(1)
    v = np.empty(1, np.uint8)
    c = np.empty(1, np.float32)
    assert lib.ps_edge_bridge_wait(ev._h, 0, v.ctypes.data, c.ctypes.data, None) == _lib.PS_EINVAL
    # an empty submission waits to empty outputs
    ev.submit(f[:0], t[:0], 0, p, slot=0)
    v, c, k = ev.wait(0)
    assert v.size == 0 and c.size == 0 and k.size == 0
    ev.close()


def test_bridge_host_input_views(w2):
    """Edges written into the numpy views of the pinned mirrors go in without
    staging and give the same bits as the same edges passed as plain arrays."""
    wl, b, sc = w2
    E = 4096
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    ev = api.EdgeEvalGpu(7, E, sc, b)
    mf, mt = ev.host_inputs()
    assert mf.shape == (E, 7) and mt.shape == (E, 7) and mf.dtype == np.float32
    for n in (E, 1000):
        mf[:n] = wl["from"][:n]
        mt[:n] = wl["to"][:n]
        v, c, _ = ev.evaluate(mf, mt, n, p)
        rv, rc, _ = ev.evaluate(np.ascontiguousarray(wl["from"][:n]), np.ascontiguousarray(wl["to"][:n]), n, p)
        np.testing.assert_array_equal(v, rv)
        assert np.array_equal(_bits(c), _bits(rc))
    ev.close()
