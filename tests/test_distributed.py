"""CPU: the multi-rank sharding logic with gloo ranks (world size 2).

Each rank runs the product's check_edges_sharded on its contiguous shard of
an edge batch, with the CPU oracle as the per-shard checker in place of the
GPU kernel that the ranks would call on their own devices, and the gathered
result must equal the unsharded one, in order.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from prismplan_b200.distributed import require_same_device, shard_range


def test_shard_range_covers_exactly():
    for n in (0, 1, 7, 64, 65537):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1


def test_model_device_mismatch_is_refused():
    require_same_device(0, 0)
    with pytest.raises(ValueError, match="built on cuda:1 but cuda:0"):
        require_same_device(1, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    import oracle
    from prismplan_b200 import workloads
    from prismplan_b200.distributed import check_edges_sharded
    from prismplan_b200.robot import RobotModelBuilder

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl = workloads.workload(2, scale=1.0 / 256)
        om = oracle.OracleModel(RobotModelBuilder.from_asset(wl["asset"]), *wl["obbs"])
        frm, to, G = wl["from"], wl["to"], np.minimum(wl["G"], 40)

        seen = []

        def checker(f, t, g):
            seen.append(len(f))
            v, c, _, _, _ = om.check_edges(f, t, g, threads=1)
            return v, c

        valid, cost = check_edges_sharded(None, None, frm, to, samples=G, checker=checker)
        assert seen == [128], seen   # this rank's half only
        if rank == 0:
            v_all, c_all, _, _, _ = om.check_edges(frm, to, G, threads=1)
            q.put((bool(np.array_equal(valid, v_all)), bool(np.array_equal(cost, c_all)), len(valid)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_gloo_two_ranks_gather_equals_single():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    same_valid, same_cost, n = q.get(timeout=5)
    assert same_valid and same_cost and n == 256
