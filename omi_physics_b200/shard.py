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


def shard_requests(requests: Sequence[dict], rank: int, world_size: int) -> List[int]:
    """Indices of the serving requests this rank admits: the same LPT plan
    over the requests' body counts, so one request stream is split across
    GPUs without any rank seeing another's worlds."""
    return local_shard([int(r['bodies']) for r in requests], rank, world_size)


class ShardedWorlds:
    """One fixed list of worlds split across ranks: this rank's shard stepped
    as :class:`~omi_physics_b200.groups.WorldGroups` on its own GPU.

    ``body_counts`` are every world's body counts and ``build(i)`` returns
    world ``i`` and its dt; each rank builds only its own worlds. ``indices``
    are the global indices of the local worlds (ascending). Every rank
    computes the same plan from the body counts, so nothing is exchanged to
    build it, and stepping involves no collective: only the host-side
    bookkeeping (the job's step time, totals, merged tick latencies) crosses
    ranks.
    """

    def __init__(self, body_counts: Sequence[int], build, rank: int, world_size: int,
                 groups: int = 4, device: int = 0, load: bool = True):
        self.rank, self.world_size = rank, world_size
        self.plan = plan_shards(body_counts, world_size)
        self.indices = self.plan[rank]
        built = [build(i) for i in self.indices]
        self.worlds = [w for w, _ in built]
        self.dts = [dt for _, dt in built]
        self.local_bodies = int(sum(int(np.count_nonzero(w.motion_type == 2)) for w in self.worlds))
        self.groups = None
        if load and self.worlds:
            from .groups import WorldGroups
            self.groups = WorldGroups(self.worlds, dts=self.dts, groups=groups, device=device)

    def step(self, n: int = 1) -> None:
        if self.groups is not None:
            self.groups.step(n)

    def close(self) -> None:
        if self.groups is not None:
            self.groups.close()


def merge_ticks(ticks: Sequence[float], world_size: int) -> List[float]:
    """Per-tick latency of the job from each rank's per-tick latencies: a
    tick ends when its slowest rank's does (element-wise max over ranks)."""
    if world_size == 1:
        return [float(t) for t in ticks]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x) for x in ticks], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().tolist()


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
