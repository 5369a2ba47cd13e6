"""Work distribution over GPUs for independent solves (batched patches, served
requests): one process per GPU, no device collective on the data path.

Units are assigned to ranks greedily by algorithmic bytes (largest first onto the
least loaded rank), the same on every rank because the assignment depends only on
the unit costs.  Results are gathered on the host through torch.distributed (NCCL
between GPUs, gloo for CPU tests), and timings are reduced as the maximum over
ranks.
"""
from __future__ import annotations

import numpy as np


def assign(costs, world: int):
    """Rank of each unit: longest-processing-time-first greedy on the costs (ties
    broken by unit index, so every rank computes the same assignment)."""
    costs = [float(c) for c in costs]
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return owner


def loads(costs, owner, world: int):
    out = [0.0] * world
    for c, r in zip(costs, owner):
        out[r] += float(c)
    return out


def max_over_ranks(x: float, group=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_results(local: dict, group=None) -> dict:
    """Merge {unit index: numpy array} dictionaries of all ranks on every rank."""
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, {k: np.asarray(v) for k, v in local.items()}, group=group)
    out = {}
    for p in parts:
        out.update(p)
    return out
