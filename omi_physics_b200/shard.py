"""Worlds across GPUs: whole worlds per rank, no data-path collective.

Independent worlds never exchange anything, so a multi-GPU job is one
process per GPU, each owning a disjoint set of whole worlds (body-count LPT
bin-packing), stepping them with its own arena. The only cross-rank traffic
is bookkeeping: the step time (max over ranks, the job's time), body counts
and tick statistics (sums / gathers), done through ``torch.distributed``
(NCCL on GPUs, gloo on CPU - the reductions are the same code).
A single world is not split: it runs as replicas.
"""
from typing import List, Sequence

import numpy as np


def plan_shards(body_counts: Sequence[int], n_ranks: int) -> List[List[int]]:
    """Longest-processing-time assignment of worlds to ranks by body count.

    Worlds in descending body count (ties: lower index first) each go to the
    rank with the fewest bodies so far (ties: lower rank). Deterministic, so
    every rank computes the same plan without communicating. Each shard lists
    its worlds in ascending index order.
    """
    if n_ranks < 1:
        raise ValueError('n_ranks must be >= 1')
    counts = np.asarray(body_counts, dtype=np.int64)
    order = sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i))
    load = [0] * n_ranks
    shards: List[List[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += int(counts[i])
    return [sorted(s) for s in shards]


def local_shard(body_counts: Sequence[int], rank: int, world_size: int) -> List[int]:
    return plan_shards(body_counts, world_size)[rank]


def _device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == 'nccl':
        return torch.device('cuda', torch.cuda.current_device())
    return torch.device('cpu')


def _reduce(x: float, op_name: str, world_size: int) -> float:
    if world_size == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x: float, world_size: int) -> float:
    """The job's time for a step: the slowest rank's."""
    return _reduce(x, 'MAX', world_size)


def sum_over_ranks(x: float, world_size: int) -> float:
    return _reduce(x, 'SUM', world_size)


def barrier(world_size: int) -> None:
    if world_size > 1:
        import torch.distributed as dist
        dist.barrier()


def gather_to_rank0(obj, world_size: int):
    """Every rank's ``obj`` as a list on rank 0 (None elsewhere)."""
    if world_size == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world_size if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
