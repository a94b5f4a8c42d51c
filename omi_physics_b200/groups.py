"""Independent worlds on one GPU as several concurrently stepped groups.

A :class:`WorldBatch` advances all its worlds stage by stage: every stage
waits for the slowest world before the next starts. Worlds never interact,
so splitting them into groups - one context, arena and CUDA stream each -
lets one group's slow stage (the contact sweep of its largest world)
overlap the other groups' broadphase, narrowphase and prep, and lets one
group's host<->device copies overlap another group's kernels.

Groups are balanced by body count (worlds in descending size dealt out in a
snake order). Stepping from the host uses one thread per group (the C ABI
releases the GIL and each context belongs to one thread); ``step_async`` +
``sync`` enqueue on all groups' streams from the calling thread.
"""
from concurrent.futures import ThreadPoolExecutor
from typing import List, Optional, Sequence

import numpy as np

from ._lib import D, U8, ptr
from .batch import WorldBatch


def plan_groups(body_counts: Sequence[int], groups: int) -> List[List[int]]:
    """World indices per group: descending size, dealt 0..G-1, G-1..0, ..."""
    order = sorted(range(len(body_counts)), key=lambda i: (-int(body_counts[i]), i))
    out: List[List[int]] = [[] for _ in range(groups)]
    for j, i in enumerate(order):
        r = j % (2 * groups)
        out[r if r < groups else 2 * groups - 1 - r].append(i)
    return [sorted(g) for g in out if g]


class WorldGroups:
    """``worlds`` split into ``groups`` batches stepped concurrently on one GPU.

    ``tuning='auto'`` (the default) applies the autotuner's cached entry for
    this GPU and workload (:func:`omi_physics_b200.tune.tuned_for`): its
    launch configuration, and its group count when ``groups`` is None; with
    no entry the defaults stand (4 groups). ``tuning`` may also be a dict of
    launch parameters, or None for the library defaults. ``own_streams``
    gives every group a torch stream of its own (``stream_handles``)."""

    def __init__(self, worlds: Sequence, dts: Sequence[float] = None, groups: Optional[int] = None,
                 device: int = 0, tuning='auto', own_streams: bool = False):
        self.worlds = list(worlds)
        dts = list(dts) if dts is not None else [w.fixed_dt for w in self.worlds]
        launch = None
        self.tuned = None
        if tuning == 'auto':
            from .tune import tuned_for
            self.tuned = tuned_for(self.worlds, device)
            if self.tuned is not None:
                launch = self.tuned.get('launch')
                if groups is None:
                    groups = int(self.tuned.get('groups', 4))
        elif isinstance(tuning, dict):
            launch = tuning
        if groups is None:
            groups = 4
        self.plan = plan_groups([w.body_count for w in self.worlds], max(1, groups))
        self.batches = [WorldBatch([self.worlds[i] for i in g], device=device, dts=[dts[i] for i in g])
                        for g in self.plan]
        self._pool = ThreadPoolExecutor(max_workers=max(1, len(self.batches)))
        self.stream_handles = []
        if own_streams:
            import torch
            self._streams = [torch.cuda.Stream(device=device) for _ in self.batches]
            self.set_streams([s.cuda_stream for s in self._streams])
        if launch:
            self.set_tuning(launch)
        # world index -> (group, index in group)
        self.where = {}
        for gi, g in enumerate(self.plan):
            for j, i in enumerate(g):
                self.where[i] = (gi, j)

    def __len__(self):
        return len(self.batches)

    def set_streams(self, streams: Sequence[int]) -> None:
        """Put each group's launches on the given cudaStream_t handles."""
        self.stream_handles = [int(s) for s in streams]
        for b, s in zip(self.batches, streams):
            b.ctx.call('set_stream', int(s))

    def set_tuning(self, launch: dict) -> None:
        """The same launch configuration for every group (keys of DEFAULT_TUNING)."""
        for b in self.batches:
            b.ctx.set_tuning(**launch)

    # -- stepping ---------------------------------------------------------------
    def _each(self, fn):
        return [f.result() for f in [self._pool.submit(fn, b) for b in self.batches]]

    def step(self, n: int = 1) -> None:
        """``n`` steps of every world (buffer regrowth handled per group)."""
        self._each(lambda b: b.step(n))

    def step_async(self, n: int = 1) -> None:
        """Enqueue ``n`` steps on every group's stream; ``sync`` waits (and
        raises if a group overflowed its buffers - re-run with ``step``)."""
        for b in self.batches:
            b.step_async(n)

    def sync(self) -> None:
        for b in self.batches:
            b.sync()

    def sync_to_host(self) -> None:
        self._each(lambda b: b.sync_to_host())

    # -- host state round trips ---------------------------------------------------
    def host_buffers(self, alloc=np.zeros):
        """Per group, arrays for the mutable state of all its rows (``alloc`` may
        give pinned memory): pos, q, v, w, awake, sleep timer."""
        out = []
        for b in self.batches:
            nb = b.packed.n_bodies
            out.append({'pos': alloc((nb, 3)), 'q': alloc((nb, 4)), 'v': alloc((nb, 3)),
                        'w': alloc((nb, 3)), 'awake': alloc((nb,), np.uint8), 'timer': alloc((nb,))})
        return out

    def step_from_host(self, bufs, n: int = 1, rounds: int = 1) -> None:
        """``rounds`` times per group: upload its state from ``bufs``, step ``n``
        times, download it back. The groups run concurrently and independently
        (no barrier between rounds), so one group's copies overlap the others'
        kernels."""
        def run(pair):
            b, h = pair
            nb = b.packed.n_bodies
            c = b.ctx
            for _ in range(rounds):
                c.call('upload_state', 0, nb, ptr(h['pos'], D), ptr(h['q'], D), ptr(h['v'], D), ptr(h['w'], D),
                       ptr(h['awake'], U8), ptr(h['timer'], D))
                c.call('step', int(n))
                c.call('download_state', 0, nb, ptr(h['pos'], D), ptr(h['q'], D), ptr(h['v'], D),
                       ptr(h['w'], D), ptr(h['awake'], U8), ptr(h['timer'], D), None, None)
        list(self._pool.map(run, zip(self.batches, bufs)))

    # -- results ------------------------------------------------------------------
    def batch_of(self, i: int):
        g, j = self.where[i]
        return self.batches[g], j

    def pairs(self, i: int):
        b, j = self.batch_of(i)
        return b.pairs(j)

    def counts(self):
        W = len(self.worlds)
        p = np.zeros(W, np.int64)
        c = np.zeros(W, np.int64)
        for g, b in zip(self.plan, self.batches):
            bp, bc = b.counts()
            p[g] = bp
            c[g] = bc
        return p, c

    def launches(self) -> int:
        return sum(b.ctx.launches() for b in self.batches)

    def close(self):
        """Stop the host threads and release every group's context."""
        self._pool.shutdown(wait=True)
        for b in self.batches:
            b.ctx.close()
