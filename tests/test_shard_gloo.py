"""Ensemble work division and the max-over-ranks timing reduction, exercised
with two gloo ranks on CPU (the multi-GPU path of the benchmark uses the same
helpers over NCCL)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from semiimplicitfv_b200.shard import max_over_ranks, partition_by_cost, rank_share, sum_over_ranks


def _costs(count=2048, seed=0):
    rng = np.random.default_rng(seed)
    n = np.round(np.exp(rng.uniform(np.log(256), np.log(16384), count)))
    return (n * n).tolist()


def test_partition_is_disjoint_complete_and_balanced():
    costs = _costs()
    for world in (1, 2, 3, 4, 8):
        parts = partition_by_cost(costs, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[k] for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-9
        assert max(loads) <= sum(costs) / world + max(costs)


def test_partition_is_deterministic():
    costs = _costs(seed=3)
    assert partition_by_cost(costs, 4) == partition_by_cost(list(costs), 4)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        share = rank_share(costs, rank, world)
        # every rank derives the same division independently: check by gathering
        gathered = [None] * world
        dist.all_gather_object(gathered, share)
        flat = sorted(k for p in gathered for k in p)
        ok_cover = flat == list(range(len(costs)))
        mine = float(sum(costs[k] for k in share))
        worst = max_over_ranks(mine)
        total = sum_over_ranks(mine)
        out.put((rank, ok_cover, mine, worst, total))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_ensemble():
    costs = _costs(count=300, seed=5)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert all(r[1] for r in res)
    loads = [r[2] for r in res]
    assert all(r[3] == max(loads) for r in res)
    assert all(abs(r[4] - sum(costs)) <= 1e-6 * sum(costs) for r in res)
