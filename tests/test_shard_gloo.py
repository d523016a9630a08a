"""Multi-process host logic of the multi-GPU batched run, on CPU with the gloo backend.

Two ranks partition the 256-instance batched distribution by the LPT rule, gather their shares and
a per-rank time: the shares must be disjoint and complete, balanced, identical on both ranks, and
the gathered time the maximum over ranks.  No GPU is involved; the instances themselves are never
built here.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from ugks2d_high_order_b200.case import batched_cases
    from ugks2d_high_order_b200.shard import instance_cost, max_over_ranks, shard, sum_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        cases = batched_cases()
        costs = [instance_cost(c, n * n) for c, n in cases]
        mine, idx = shard(cases, costs, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, idx)
        load = sum(costs[i] for i in idx)
        total = sum_over_ranks(load, dist)
        tmax = max_over_ranks(1.0 + rank, dist)     # a stand-in per-rank time
        out[rank] = {"gathered": gathered, "load": load, "total": total, "tmax": tmax, "n": len(mine)}
    finally:
        dist.destroy_process_group()


def test_lpt_shards_partition_the_batch_over_two_gloo_ranks():
    from ugks2d_high_order_b200.case import batched_cases
    from ugks2d_high_order_b200.shard import instance_cost
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    cases = batched_cases()
    costs = [instance_cost(c, n * n) for c, n in cases]
    g0, g1 = res[0]["gathered"], res[1]["gathered"]
    assert g0 == g1                                       # every rank sees the same partition
    allidx = sorted(g0[0] + g0[1])
    assert allidx == list(range(len(cases)))              # disjoint and complete
    loads = [res[r]["load"] for r in range(world)]
    assert sum(loads) == sum(costs) == res[0]["total"] == res[1]["total"]
    assert max(loads) / min(loads) < 1.01                 # LPT balance on 256 uneven instances
    assert res[0]["tmax"] == res[1]["tmax"] == 2.0        # max over ranks


@pytest.mark.parametrize("nparts", [1, 3, 8])
def test_lpt_partition_is_complete_and_balanced(nparts):
    from ugks2d_high_order_b200.shard import lpt_partition
    costs = [5, 9, 2, 7, 7, 1, 3, 8, 6, 4] * 5
    part = lpt_partition(costs, nparts)
    loads = [sum(c for c, p in zip(costs, part) if p == b) for b in range(nparts)]
    assert sum(loads) == sum(costs) and len(part) == len(costs)
    assert max(loads) - min(loads) <= max(costs)
