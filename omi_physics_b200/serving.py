"""Continuous-batching request loop over device-resident worlds.

A :class:`Server` reserves arenas of *slots* in size classes (per-slot
capacities, ``omi_reserve_slots_each``) under an HBM budget
(``omi_set_budget``: a reservation fails with :class:`OutOfBudget` above it).
Requests - a world plus a step count - queue on arrival. Every tick:

1. admit queued requests that have arrived, in arrival order, each into the
   smallest free slot whose capacities hold it (``omi_load_world``: no
   reallocation, no graph rebuild - the other slots keep stepping). With a
   budget, a request whose classes are all full does not wait for a slot:
   the server reserves a new *chunk* (one more context and arena of
   ``chunk_slots`` slots of the smallest class that holds it) while the
   budget has room, so a request waits only when HBM, not a class, is full.
   Chunks are reserved whole and never resized, so admission into them
   keeps the no-reallocation property;
2. step every active slot once: each chunk's worlds in the same launches
   (its captured CUDA graph), the chunks on their own streams concurrently;
3. retire worlds whose steps are done: their rows are copied back into the
   request's world columns and the slot is freed.

Worlds never interact, so a world's result does not depend on what else is
resident: stepping it here gives the same state as stepping it alone.

The admission policy (:class:`SlotPool`) is plain Python so it can be tested
without a GPU.
"""
import bisect
import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from ._lib import (D, I, OMI_E_STATE, OMI_E_UNSUPPORTED, U8, Context, OmiError, OmiSlotCaps,
                   UnsupportedFeature, ptr)
from .arena import pack_worlds


@dataclass(frozen=True)
class SlotClass:
    """``count`` slots, each able to hold a world within these capacities."""
    bodies: int
    count: int
    shapes: int = -1            # -1: same as bodies
    materials: int = -1         # -1: same as bodies
    points: int = 0
    joints: int = 0
    filter_rows: int = 8
    pair_friction: int = 16

    def caps(self) -> OmiSlotCaps:
        return OmiSlotCaps(self.bodies, self.shapes if self.shapes >= 0 else self.bodies,
                           self.materials if self.materials >= 0 else self.bodies, self.points,
                           self.joints, self.filter_rows, self.pair_friction)


def need_of(scene) -> tuple:
    """Capacities one packed single-world scene needs, in OmiSlotCaps order."""
    return (int(scene.n_bodies), int(scene.n_shapes), int(scene.n_materials), int(scene.n_points),
            int(scene.n_joints), int(scene.w_filter_rows[0]), int(scene.n_pair_friction))


def fits(caps: OmiSlotCaps, need: tuple) -> bool:
    have = (caps.bodies, caps.shapes, caps.materials, caps.points, caps.joints, caps.filter_rows,
            caps.pair_friction)
    return all(n <= h for n, h in zip(need, have))


def size_classes(max_bodies: int, per_class: int, min_bodies: int = 32, **kw) -> List[SlotClass]:
    """Power-of-two body classes (plus one row for a ground body) up to ``max_bodies``."""
    out, b = [], min_bodies
    while True:
        out.append(SlotClass(bodies=b + 1, count=per_class, **kw))
        if b >= max_bodies:
            return out
        b *= 2


class SlotPool:
    """Free slots per class; a request takes the smallest free slot that fits."""

    def __init__(self, caps: Sequence[OmiSlotCaps]):
        self.caps = []
        self._order = []                         # slots by capacity
        self._bodies = []
        self.free = set()
        self.add(caps)

    def add(self, caps: Sequence[OmiSlotCaps], first: Optional[int] = None) -> List[int]:
        """Append slots (ids from ``first``, default the next free id); they start free."""
        first = len(self.caps) if first is None else first
        if first != len(self.caps):
            raise ValueError('slot ids must be contiguous')
        self.caps.extend(caps)
        ids = list(range(first, first + len(caps)))
        self._order = sorted(range(len(self.caps)), key=lambda s: (self.caps[s].bodies, s))
        self._bodies = [self.caps[s].bodies for s in self._order]
        self.free.update(ids)
        return ids

    def take(self, need: tuple) -> Optional[int]:
        """A free slot holding ``need`` (smallest capacity first), or None."""
        start = bisect.bisect_left(self._bodies, need[0])
        for j in range(start, len(self._order)):
            s = self._order[j]
            if s in self.free and fits(self.caps[s], need):
                self.free.discard(s)
                return s
        return None

    def give_back(self, slot: int) -> None:
        if slot in self.free:
            raise ValueError('slot %d is already free' % slot)
        self.free.add(slot)

    def could_ever_fit(self, need: tuple) -> bool:
        return any(fits(c, need) for c in self.caps)


@dataclass
class Request:
    """One simulation request: ``steps`` steps of ``world`` at ``dt``."""
    rid: int
    world: object
    steps: int
    dt: float
    arrival: float = 0.0
    packed: object = None
    need: tuple = ()
    bodies: int = 0                 # dynamic bodies (the body-steps it contributes per step)
    slot: int = -1
    admitted_at: float = -1.0
    finished_at: float = -1.0
    done: int = 0


@dataclass
class ServeStats:
    ticks: int = 0
    tick_ms: List[float] = field(default_factory=list)      # wall time of each tick
    step_ms: List[float] = field(default_factory=list)      # device time of each tick's step
    body_steps: int = 0
    wall_s: float = 0.0
    completed: int = 0
    peak_active: int = 0
    wait_ms: List[float] = field(default_factory=list)      # arrival -> admission
    device_bytes: int = 0
    chunks_added: int = 0                                     # slot chunks reserved on demand

    def summary(self) -> dict:
        def pct(xs, q):
            return float(np.percentile(xs, q)) if len(xs) else None
        return {
            'ticks': self.ticks, 'completed': self.completed, 'peak_active': self.peak_active,
            'body_steps': self.body_steps, 'wall_s': self.wall_s,
            'body_steps_per_s': self.body_steps / self.wall_s if self.wall_s > 0 else 0.0,
            'tick_ms_p50': pct(self.tick_ms, 50), 'tick_ms_p99': pct(self.tick_ms, 99),
            'step_ms_p50': pct(self.step_ms, 50), 'step_ms_p99': pct(self.step_ms, 99),
            'wait_ms_p50': pct(self.wait_ms, 50), 'wait_ms_p99': pct(self.wait_ms, 99),
            'device_bytes': self.device_bytes, 'chunks_added': self.chunks_added,
        }


class _Chunk:
    """One context holding slots: an arena reserved once, never resized."""

    def __init__(self, caps: Sequence[OmiSlotCaps], device: int, budget: Optional[int], stream=None):
        self.ctx = Context(device)
        if stream is not None:
            self.ctx.call('set_stream', stream)
        if budget is not None:
            self.ctx.call('set_budget', max(int(budget), 1))
        arr = (OmiSlotCaps * len(caps))(*caps)
        try:
            self.ctx.call('reserve_slots_each', len(caps), arr)
            self.ctx.call('step', 1)            # capture the step graph while every slot is empty
        except Exception:
            self.ctx.close()
            raise
        self.W = len(caps)
        self.active = np.zeros(self.W, np.uint8)
        self.n_active = 0


class Server:
    """Slots in HBM, requests admitted as slots free up, one step per tick.

    ``budget_bytes`` bounds the device memory of all chunks together; with
    ``grow`` (default: on when a budget is given) full classes spill into new
    chunks of ``chunk_slots`` slots (default: each class's initial count)
    while the budget allows."""

    def __init__(self, classes: Sequence[SlotClass], device: int = 0,
                 budget_bytes: Optional[int] = None, stream=None, grow: Optional[bool] = None,
                 chunk_slots: Optional[int] = None):
        self.device = device
        self.budget = int(budget_bytes) if budget_bytes else None
        self.grow = (self.budget is not None) if grow is None else bool(grow)
        self.classes = sorted(classes, key=lambda c: c.bodies)
        self.chunk_slots = chunk_slots
        self.stream = stream
        self.chunks: List[_Chunk] = []
        self._where: List[tuple] = []          # global slot -> (chunk, local slot)
        self._cant_grow = set()                # classes whose next chunk did not fit the budget
        self.pool = SlotPool([])
        caps = [c.caps() for c in classes for _ in range(c.count)]
        self._add_chunk(caps, stream)
        self.ctx = self.chunks[0].ctx
        self.resident: Dict[int, Request] = {}
        self.queue: List[Request] = []
        self.finished: Dict[int, Request] = {}
        self.stats = ServeStats(device_bytes=self.device_bytes())
        self._next_rid = 0
        self._events = None

    @property
    def W(self) -> int:
        return len(self._where)

    def device_bytes(self) -> int:
        return sum(ch.ctx.device_bytes() for ch in self.chunks)

    def _add_chunk(self, caps, stream=None) -> None:
        left = None if self.budget is None else self.budget - self.device_bytes()
        ch = _Chunk(caps, self.device, left, stream)
        c = len(self.chunks)
        self.chunks.append(ch)
        first = len(self._where)
        self._where.extend((c, s) for s in range(ch.W))
        self.pool.add(caps, first)

    def _grow_for(self, need: tuple) -> bool:
        """Reserve a chunk of the smallest class that holds ``need``, if the
        budget has room; False when it has not (the request waits)."""
        from ._lib import OutOfBudget
        for cl in self.classes:
            if not fits(cl.caps(), need):
                continue
            if cl.bodies in self._cant_grow:
                return False
            n = self.chunk_slots or cl.count
            try:
                self._add_chunk([cl.caps()] * n)
            except OutOfBudget:
                self._cant_grow.update(c.bodies for c in self.classes if c.bodies >= cl.bodies)
                return False
            self.stats.device_bytes = self.device_bytes()
            self.stats.chunks_added += 1
            return True
        return False

    def _at(self, slot: int):
        c, s = self._where[slot]
        return self.chunks[c], s

    # -- requests ---------------------------------------------------------------
    def submit(self, world, steps: int, dt: float = None, arrival: float = 0.0) -> Request:
        dt = float(world.fixed_dt if dt is None else dt)
        packed = pack_worlds([world], [dt], active=True)
        if packed.has_sensors or packed.scene.n_volumes or packed.scene.n_meshes:
            raise UnsupportedFeature(OMI_E_UNSUPPORTED, 'serving slots do not take sensors, gravity volumes '
                                     'or triangle meshes; step such worlds in a WorldBatch')
        req = Request(self._next_rid, world, int(steps), dt, float(arrival), packed,
                      need_of(packed.scene), int(np.count_nonzero(world.motion_type == 2)))
        if not self.pool.could_ever_fit(req.need):
            raise ValueError('request %d needs %s, larger than every slot class' % (req.rid, req.need))
        self._next_rid += 1
        i = len(self.queue)
        while i > 0 and self.queue[i - 1].arrival > req.arrival:
            i -= 1
        self.queue.insert(i, req)
        return req

    def submit_document(self, gltf: dict, steps: int, dt: float = 1.0 / 60.0, arrival: float = 0.0,
                        **build) -> Request:
        """Serve an OMI glTF document: its world (``gltf.build_world``) as a request."""
        from .gltf import build_world
        return self.submit(build_world(gltf, fixed_dt=dt, **build), steps, dt, arrival)

    def _admit(self, now: float) -> int:
        n = 0
        keep = []
        for req in self.queue:
            if req.arrival > now:
                keep.append(req)
                continue
            slot = self.pool.take(req.need)
            if slot is None and self.grow and self._grow_for(req.need):
                slot = self.pool.take(req.need)
            if slot is None:
                keep.append(req)
                continue
            ch, s = self._at(slot)
            ch.ctx.call('load_world', s, C.byref(req.packed.scene))
            req.slot, req.admitted_at = slot, now
            ch.active[s] = 1
            ch.n_active += 1
            self.resident[slot] = req
            self.stats.wait_ms.append(max(0.0, now - req.arrival) * 1e3)
            n += 1
        self.queue = keep
        return n

    def _retire(self, now: float) -> int:
        done = [s for s, r in self.resident.items() if r.done >= r.steps]
        if not done:
            return 0
        touched = set()
        for slot in done:
            req = self.resident.pop(slot)
            self._download(req)
            req.finished_at = now
            ch, s = self._at(slot)
            ch.active[s] = 0
            ch.n_active -= 1
            touched.add(id(ch))
            self.pool.give_back(slot)
            self.finished[req.rid] = req
            self.stats.completed += 1
        for ch in self.chunks:
            if id(ch) in touched:
                ch.ctx.call('set_active', ptr(ch.active, U8))
        return len(done)

    def _download(self, req: Request) -> None:
        first, n = C.c_int32(), C.c_int32()
        ch, s = self._at(req.slot)
        ch.ctx.call('world_rows', s, C.byref(first), C.byref(n))
        w = req.world
        ch.ctx.call('download_state', first.value, n.value, ptr(w._position, D),
                      ptr(w._orientation, D), ptr(w._linear_velocity, D),
                      ptr(w._angular_velocity, D), ptr(w._awake.view(np.uint8), U8),
                      ptr(w._sleep_timer, D), ptr(w._aabb_min, D), ptr(w._aabb_max, D))
        w.time += req.steps * req.dt

    # -- snapshot / restore of resident worlds -----------------------------------
    def _rows(self, slot: int):
        first, n = C.c_int32(), C.c_int32()
        ch, s = self._at(slot)
        ch.ctx.call('world_rows', s, C.byref(first), C.byref(n))
        return first.value, n.value

    def snapshot(self, req: Request) -> dict:
        """A resident request's state, warm-start cache and progress (host arrays)."""
        if req.slot < 0 or self.resident.get(req.slot) is not req:
            raise ValueError('request %d is not resident' % req.rid)
        first, n = self._rows(req.slot)
        ch, s = self._at(req.slot)
        cols = {k: np.zeros((n, d)) for k, d in (('pos', 3), ('q', 4), ('v', 3), ('w', 3))}
        awake = np.zeros(n, np.uint8)
        timer = np.zeros(n)
        ch.ctx.call('download_state', first, n, ptr(cols['pos'], D), ptr(cols['q'], D),
                    ptr(cols['v'], D), ptr(cols['w'], D), ptr(awake, U8), ptr(timer, D), None, None)
        cap = 1 << 12
        while True:
            a = np.zeros(cap, np.int32); b = np.zeros(cap, np.int32)
            pt = np.zeros((cap, 3)); imp = np.zeros((cap, 3))
            rc = ch.ctx.lib.omi_get_cache(ch.ctx.h, s, ptr(a, I), ptr(b, I), ptr(pt, D), ptr(imp, D), cap)
            if rc == -2 and cap < (1 << 26):
                cap *= 8
                continue
            k = ch.ctx.check(rc, 'omi_get_cache')
            break
        return dict(cols, awake=awake, timer=timer, done=req.done,
                    cache=dict(a=a[:k] - first, b=b[:k] - first, point=pt[:k], impulse=imp[:k]))

    def restore(self, req: Request, snap: dict) -> None:
        """Put a :meth:`snapshot` back into the request's slot; stepping on gives
        exactly what stepping on from the snapshot would have."""
        if req.slot < 0 or self.resident.get(req.slot) is not req:
            raise ValueError('request %d is not resident' % req.rid)
        first, n = self._rows(req.slot)
        ch, s = self._at(req.slot)
        pos, q, v, w = (np.ascontiguousarray(snap[k], 'd') for k in ('pos', 'q', 'v', 'w'))
        awake = np.ascontiguousarray(snap['awake'], np.uint8)
        timer = np.ascontiguousarray(snap['timer'], 'd')
        ch.ctx.call('upload_state', first, n, ptr(pos, D), ptr(q, D), ptr(v, D), ptr(w, D),
                    ptr(awake, U8), ptr(timer, D))
        c = snap['cache']
        a = np.ascontiguousarray(np.asarray(c['a'], np.int32) + first)
        b = np.ascontiguousarray(np.asarray(c['b'], np.int32) + first)
        pt = np.ascontiguousarray(c['point'], 'd').reshape(-1, 3)
        imp = np.ascontiguousarray(c['impulse'], 'd').reshape(-1, 3)
        ch.ctx.call('set_cache', s, len(a), ptr(a, I), ptr(b, I), ptr(pt, D), ptr(imp, D))
        req.done = int(snap['done'])

    # -- ticks ------------------------------------------------------------------
    def tick(self, now: float) -> None:
        """Admit, step every resident world once, retire finished ones."""
        t = time.perf_counter()
        self._admit(now)
        if self.resident:
            busy = [ch for ch in self.chunks if ch.n_active]
            ev = self._step_events() if len(self.chunks) == 1 else None
            t1 = time.perf_counter()
            if ev is not None:
                ev[0].record(self._torch_stream)
            if len(busy) == 1:
                busy[0].ctx.call('step', 1)
            else:
                for ch in busy:                 # every chunk on its own stream, concurrently
                    ch.ctx.call('step_async', 1)
                for ch in busy:
                    try:
                        ch.ctx.call('sync')
                    except OmiError as e:
                        if e.code != OMI_E_STATE:
                            raise
                        # the step found more pairs or contacts than its buffers hold and
                        # did nothing: the synchronous step regrows them and runs it
                        ch.ctx.call('step', 1)
            if ev is not None:
                ev[1].record(self._torch_stream)
                ev[1].synchronize()
                self.stats.step_ms.append(ev[0].elapsed_time(ev[1]))
            else:
                self.stats.step_ms.append((time.perf_counter() - t1) * 1e3)
            for r in self.resident.values():
                r.done += 1
                self.stats.body_steps += r.bodies
            self.stats.peak_active = max(self.stats.peak_active, len(self.resident))
            self.stats.ticks += 1
        self._retire(now)
        self.stats.tick_ms.append((time.perf_counter() - t) * 1e3)

    def _step_events(self):
        """CUDA events on the library's stream, when it is a torch stream."""
        if self._events is None:
            self._events = False
            if self.stream is not None:
                try:
                    import torch
                    self._torch_stream = torch.cuda.ExternalStream(self.stream)
                    self._events = True
                except Exception:
                    pass
        if not self._events:
            return None
        import torch
        return (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))

    def run(self, clock: str = 'wall', max_ticks: int = None) -> ServeStats:
        """Serve until every submitted request is done.

        ``clock='wall'``: arrivals are seconds after the start of the loop,
        and an idle server sleeps until the next arrival. ``clock='ticks'``:
        arrivals are tick numbers (deterministic, for tests).
        """
        t0 = time.perf_counter()
        k = 0
        while self.queue or self.resident:
            if clock == 'wall':
                now = time.perf_counter() - t0
                if not self.resident and self.queue and self.queue[0].arrival > now:
                    time.sleep(min(self.queue[0].arrival - now, 0.05))
                    continue
            else:
                now = float(k)
            self.tick(now)
            k += 1
            if max_ticks is not None and k >= max_ticks:
                break
        self.stats.wall_s = time.perf_counter() - t0
        return self.stats

    def close(self):
        for ch in self.chunks:
            ch.ctx.close()
