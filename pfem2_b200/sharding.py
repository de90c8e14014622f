"""Instance sharding for batches of independent PFEM2 instances.

A single mesh does not shard here (the path is single-GPU), but a batch of
independent instances (the ensemble workload, a parameter sweep) does: every
rank runs its own subset as one batched context, with no data-path
collective. The split is a longest-processing-time assignment on a cost per
instance (cells, or cells plus particles): instances in decreasing cost
order, each to the currently least-loaded rank. It is deterministic (ties by
instance index, then by rank), so every rank computes the same split on its
own without exchanging anything; `check_split_agrees` verifies that across a
process group.
"""
from typing import List, Sequence


def lpt_split(costs: Sequence[float], n_ranks: int) -> List[List[int]]:
    """Instance indices per rank (each list ascending)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * n_ranks
    parts: List[List[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def instance_cost(spec) -> float:
    """Work estimate of one instance: its cells times the particles per cell."""
    q = 1
    for v in spec.q:
        q *= int(v)
    return float(spec.mesh.n_cells) * (1.0 + q)


def shard(specs: Sequence, rank: int, world: int):
    """(instance indices, specs) that `rank` of `world` runs."""
    idx = lpt_split([instance_cost(s) for s in specs], world)[rank]
    return idx, [specs[i] for i in idx]


def imbalance(costs: Sequence[float], parts: Sequence[Sequence[int]]) -> float:
    """max rank load / mean rank load (1.0 = perfect)."""
    loads = [sum(costs[i] for i in p) for p in parts]
    mean = sum(loads) / max(1, len(loads))
    return max(loads) / mean if mean > 0 else 1.0


def check_split_agrees(idx: Sequence[int], n_instances: int, group=None) -> bool:
    """All-gathers every rank's instance list and checks that the lists are
    disjoint and cover 0..n_instances-1 (run on every rank of the group)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    mine = torch.full((n_instances,), -1, dtype=torch.int64)
    mine[: len(idx)] = torch.tensor(list(idx), dtype=torch.int64)
    out = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(out, mine, group=group)
    seen = sorted(int(v) for t in out for v in t.tolist() if v >= 0)
    return seen == list(range(n_instances))


def max_over_ranks(value: float, group=None) -> float:
    """The largest `value` over the ranks (timings are reported as the max)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return value
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
