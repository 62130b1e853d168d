"""Multi-GPU host logic on CPU: world_size-2 gloo ranks.

Each rank asks the library for its share of the heaviest-first work items
(hj_shard_plan, the selection hj_join applies with shard_count/shard_index);
together the shares must cover every item exactly once and stay balanced, and
the only collective the join needs -- summing per-rank pair counts and taking
the max step time -- must give the whole-job figures.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, n_items, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import hegjoin_b200 as hj
    first, stride, m = hj.shard_plan(n_items, world, rank)
    mine = list(range(first, n_items, stride))
    assert len(mine) == m
    # stand-in per-item pair counts: heaviest first, like the workload order
    pairs = sum(1000 - i for i in mine)
    sizes = [None] * world
    dist.all_gather_object(sizes, mine)
    t = torch.tensor([float(pairs), float(10 + rank)], dtype=torch.float64)
    tot = t.clone()
    dist.all_reduce(tot[:1], op=dist.ReduceOp.SUM)
    mx = t.clone()
    dist.all_reduce(mx[1:], op=dist.ReduceOp.MAX)
    if rank == 0:
        q.put((sizes, tot[0].item(), mx[1].item()))
    dist.destroy_process_group()


@pytest.mark.parametrize("n_items", [0, 1, 7, 1000])
def test_two_rank_shards_cover_all_items(n_items):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, n_items, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    sizes, tot, mx = q.get(timeout=10)
    allv = sorted(sizes[0] + sizes[1])
    assert allv == list(range(n_items))
    assert abs(len(sizes[0]) - len(sizes[1])) <= 1
    assert tot == sum(1000 - i for i in range(n_items))
    assert mx == 11.0


def test_shard_plan_rejects_bad_index():
    import hegjoin_b200 as hj
    with pytest.raises(hj.HJError):
        hj.shard_plan(10, 2, 2)


# ---- greedy LPT: the partition hj_join applies with shard_count > 1 ---------------------------
def _lpt_rank(rank, world, port, costs, q):
    import numpy as np
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import hegjoin_b200 as hj
    mine = hj.shard_plan_lpt(np.array(costs, np.uint64), world, rank).tolist()
    parts = [None] * world
    dist.all_gather_object(parts, mine)
    if rank == 0:
        q.put(parts)
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_lpt_ranks_partition_items_and_balance(world):
    import numpy as np
    rng = np.random.default_rng(world)
    costs = (rng.pareto(1.2, 500) * 1000).astype(np.uint64).tolist()   # skewed item costs
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_lpt_rank, args=(r, world, port, costs, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    parts = q.get(timeout=10)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))     # every item exactly once
    loads = [sum(costs[i] for i in p) for p in parts]
    # Graham's bound for LPT: the largest load is within max(cost) of the mean
    assert max(loads) - sum(loads) / world <= max(costs)
    for p in parts:
        assert p == sorted(p)


def test_lpt_plan_cases():
    import numpy as np
    import hegjoin_b200 as hj
    c = np.array([5, 4, 3, 3, 2, 1], np.uint64)
    assert hj.shard_plan_lpt(c, 2, 0).tolist() == [0, 3, 5]
    assert hj.shard_plan_lpt(c, 2, 1).tolist() == [1, 2, 4]
    assert hj.shard_plan_lpt(np.zeros(0, np.uint64), 2, 1).tolist() == []
    assert hj.shard_plan_lpt(c, 1, 0).tolist() == list(range(6))
    assert hj.shard_plan_lpt(c, 8, 7).tolist() == []                  # more ranks than items
    with pytest.raises(hj.HJError):
        hj.shard_plan_lpt(c, 2, 2)
