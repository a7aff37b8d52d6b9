"""Instance sharding across ranks (one process per GPU, torch.distributed).

Batched instances are independent, so a batch shards by instance with no
collective on the forward data path.  The one exchange step is the adjoint's
weight gradient, summed over every rank's instances (allreduce_weight_grads);
the bench also takes the max over ranks of its measured times.  Two layouts:

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


def allreduce_weight_grads(grad_qd, grad_r, grad_q_ee):
    """The adjoint's exchange step for data-parallel tuning of the cost weights: each rank sums
    gpt_sqp_adjoint's per-instance gradients over its instances (grad_qd [B, 7], grad_r [B, 7],
    grad_q_ee [B]), and one all-reduce (sum) over the ranks of the packed 15 numbers gives every
    rank the gradient of the whole batch.  Returns the packed float64 vector [qd (7), r (7), q_ee]
    on the inputs' device (the rank's own sums without a process group)."""
    import torch
    import torch.distributed as dist
    packed = torch.cat([grad_qd.reshape(-1, 7).sum(0), grad_r.reshape(-1, 7).sum(0),
                        grad_q_ee.reshape(-1).sum().reshape(1)]).to(torch.float64)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(packed, op=dist.ReduceOp.SUM)
    return packed
