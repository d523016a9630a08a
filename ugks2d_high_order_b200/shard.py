"""Sharding of independent Couette instances across GPUs (one process per GPU).

Instances never exchange data, so a multi-GPU batched run is a partition of the instances plus a
host-side gather of the metric: no collective on the data path.  The partition is a
largest-processing-time greedy on each instance's cost (cells x velocities), the same rule
the batch runtime uses for its stream slots.
"""
import numpy as np


def instance_cost(case, nvel):
    """Work of one S2CN2 step of an instance: cells x velocities."""
    return case.nx * case.ny * nvel


def lpt_partition(costs, nparts):
    """Assign items to nparts bins, largest first, each to the least-loaded bin (ties: lowest bin).
    Returns the bin of every item."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = np.zeros(nparts)
    part = [0] * len(costs)
    for i in order:
        b = int(np.argmin(load))
        part[i] = b
        load[b] += costs[i]
    return part


def shard(items, costs, rank, world):
    """The items rank `rank` of `world` runs, in their original order, and their indices."""
    part = lpt_partition(costs, world)
    idx = [i for i, p in enumerate(part) if p == rank]
    return [items[i] for i in idx], idx


def max_over_ranks(x, pg=None, device=None):
    """The maximum of a per-rank float over the process group (the slowest rank's time)."""
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, pg=None, device=None):
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())
