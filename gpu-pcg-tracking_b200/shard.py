"""Instance sharding across ranks (one process per GPU, torch.distributed).

Batched instances are independent, so a batch shards by instance with no
collective on the data path; the only collective is the max over ranks of the
measured times.  Two layouts:

* weak scaling (the bench): every rank solves `per_rank` instances of its own,
  global instance ids rank * per_rank + i (the problem generator's seeds);
* a fixed global batch of uneven horizons: instances sorted by horizon
  (longest first) and dealt round-robin, so every rank gets about the same
  number of knots.
"""
from typing import List, Sequence


def weak_scaling_ids(rank: int, world: int, per_rank: int) -> List[int]:
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return list(range(rank * per_rank, (rank + 1) * per_rank))


def shard_instances(knot_points: Sequence[int], rank: int, world: int) -> List[int]:
    """Indices (ascending) of the instances rank `rank` of `world` solves."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    order = sorted(range(len(knot_points)), key=lambda i: (-knot_points[i], i))
    return sorted(i for j, i in enumerate(order) if j % world == rank)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over the ranks of the default process group (the value itself
    without one).  `device` is where the reduction tensor lives (cuda for NCCL, cpu for gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
