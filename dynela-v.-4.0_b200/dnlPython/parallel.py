"""Several GPUs, one process per GPU: independent models (a batch of
simulations) are partitioned across the ranks with no exchange during the
run; a single mesh runs as one replica per rank.  The only collectives are
the timing barrier, the max-over-ranks of the measured times and, at the
end, one gather of the per-instance result records (a few bytes each)
(torch.distributed: NCCL on GPUs, gloo on the host).
"""
import numpy as np


def instance_cost(desc):
    """Work estimate of one instance run to its end time: elements x
    increments, the increment count growing like the inverse element size,
    i.e. like n_elems^(1/3) for a fixed geometry."""
    return float(desc.n_elems) ** (4.0 / 3.0)


def shard_instances(costs, world):
    """Longest-processing-time partition of instances over `world` ranks:
    instances in decreasing cost, each to the least loaded rank (ties to the
    lowest rank).  Deterministic; returns one sorted index list per rank."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = np.zeros(world)
    parts = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def reduce_max(value, dist, device=None):
    """Max of a float over the ranks (value itself without a process group)."""
    if dist is None:
        return value
    import torch
    if device is None:
        device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value, dist, device=None):
    """Sum of a float over the ranks."""
    if dist is None:
        return value
    import torch
    if device is None:
        device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_records(records, dist):
    """Per-instance result records of every rank, merged on every rank:
    `records` maps this rank's instance indices to small dicts; returns one
    dict of all instances (records of the same index from two ranks are an
    error: the partition gives each instance to one rank)."""
    if dist is None:
        return dict(records)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(records))
    out = {}
    for p in parts:
        for k, v in p.items():
            if k in out:
                raise ValueError(f"instance {k} reported by two ranks")
            out[k] = v
    return out
