"""Work division across ranks (one process per GPU).

The explicit step, the semi-implicit step and the adjoint run one problem per
GPU (replicas); an ensemble of independent problems is divided across ranks
by estimated cost with no data-path exchange: a tube of n cells costs ~ n^2
(cells x steps, steps ~ n at a fixed CFL), and a greedy longest-first
assignment to the least-loaded rank keeps the ranks within one tube's cost of
each other.
"""
from __future__ import annotations

from typing import List, Sequence


def partition_by_cost(costs: Sequence[float], nparts: int) -> List[List[int]]:
    """Indices of `costs` split into `nparts` lists (longest processing time
    first; ties broken by index, so every rank computes the same split)."""
    if nparts <= 0:
        raise ValueError("nparts must be positive")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    loads = [0.0] * nparts
    parts: List[List[int]] = [[] for _ in range(nparts)]
    for k in order:
        r = min(range(nparts), key=lambda q: (loads[q], q))
        parts[r].append(k)
        loads[r] += float(costs[k])
    return [sorted(p) for p in parts]


def rank_share(costs: Sequence[float], rank: int, world: int) -> List[int]:
    return partition_by_cost(costs, world)[rank]


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of a per-rank scalar over the default process group (NCCL with
    a CUDA device, gloo on CPU); the value itself without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
