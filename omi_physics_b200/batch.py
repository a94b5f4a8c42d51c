"""Device-resident worlds: the batched form and the state shuttle the plain
backend uses.

:class:`WorldBatch` loads any number of independent worlds (reference
``PhysicsWorld`` layout) into one device arena and steps them all with the
same launches — one CUDA graph per step for every world, whatever their
sizes. State stays in HBM between steps; :meth:`WorldBatch.sync_to_host`
writes it back into each world's numpy columns.
"""
import ctypes as C
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from ._lib import D, I, U8, Context, ptr
from .arena import pack_worlds, world_flags, world_iterations
from .joints import joint_kind


@dataclass
class Contact:
    """One contact record (collide.py:37-53): normal points from ``a`` to ``b``."""
    a: int
    b: int
    point: np.ndarray
    normal: np.ndarray
    depth: float
    normal_impulse: float = 0.0
    tangent_impulse: np.ndarray = field(default_factory=lambda: np.zeros(2))


class WorldBatch:
    """Independent worlds stepped together on one GPU."""

    def __init__(self, worlds: Sequence, device: int = 0, dts: Sequence[float] = None,
                 ctx: Context = None):
        self.worlds = list(worlds)
        self.ctx = ctx or Context(device)
        self.dts = list(dts) if dts is not None else [w.fixed_dt for w in self.worlds]
        self.packed = pack_worlds(self.worlds, self.dts)
        self.ctx.call('load', C.byref(self.packed.scene))
        self.offsets = self.packed.body_off
        self.joint_offsets = self.packed.joint_off
        # sensor overlaps of the last step per world and the enter / stay /
        # exit events of every step since the last take_events()
        self.has_sensors = bool(getattr(self.packed, 'has_sensors', False))
        self._sensor_worlds = [i for i, w in enumerate(self.worlds)
                               if np.any(np.asarray(w._trigger_shape[:w.body_count]) >= 0)]
        self.overlaps = [set() for _ in self.worlds]
        self.events = [[] for _ in self.worlds]

    # -- stepping -----------------------------------------------------------
    def step(self, n: int = 1) -> None:
        """``n`` steps of every active world (capacity regrowth handled inside).
        With sensors present the steps run one at a time, so each step's
        trigger events are recorded (:meth:`take_events`)."""
        if self.has_sensors:
            for _ in range(int(n)):
                self.ctx.call('step', 1)
                self._record_events()
        else:
            self.ctx.call('step', int(n))
        for w, dt in zip(self.worlds, self.dts):
            w.time += n * dt

    def trigger_overlaps(self, i: int) -> set:
        """The last step's (trigger, other) overlaps of world ``i`` (world-local
        indices), as the reference's ``TriggerSystem.overlaps`` holds them."""
        if not self.has_sensors:
            return set()
        cap = 256
        while True:
            t = np.zeros(cap, np.int32)
            o = np.zeros(cap, np.int32)
            m = self.ctx.call('get_trigger_overlaps', i, ptr(t, I), ptr(o, I), cap)
            if m <= cap:
                return {(int(a), int(b)) for a, b in zip(t[:m], o[:m])}
            cap = m

    def _record_events(self) -> None:
        """Enter / stay / exit of one step (triggers.py:36-42), sorted within
        each kind."""
        for i in self._sensor_worlds:
            new = self.trigger_overlaps(i)
            old = self.overlaps[i]
            if new or old:
                self.events[i].extend([('enter',) + p for p in sorted(new - old)] +
                                      [('stay',) + p for p in sorted(new & old)] +
                                      [('exit',) + p for p in sorted(old - new)])
            self.overlaps[i] = new

    def take_events(self, i: int) -> list:
        """World ``i``'s trigger events since the last call, oldest first."""
        ev, self.events[i] = self.events[i], []
        return ev

    def step_async(self, n: int = 1) -> None:
        """Enqueue ``n`` steps without waiting (``sync`` reports an overflow).
        Trigger events are not recorded on this path; ``trigger_overlaps``
        still gives the last step's overlaps."""
        self.ctx.call('step_async', int(n))

    def sync(self) -> None:
        self.ctx.call('sync')

    def set_active(self, mask: Sequence[bool]) -> None:
        a = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8))
        self.ctx.call('set_active', ptr(a, U8))

    def refresh_params(self) -> None:
        """Push dt, iteration counts and flags read from the world objects."""
        dt = np.array(self.dts, 'd')
        it = np.array([world_iterations(w) for w in self.worlds], np.int32)
        jit = np.array([int(w.joint_iterations) for w in self.worlds], np.int32)
        fl = np.array([world_flags(w) for w in self.worlds], np.int32)
        self.ctx.call('set_world_params', ptr(dt, D), ptr(it, I), ptr(jit, I), ptr(fl, I))

    # -- state ------------------------------------------------------------------
    def upload_state(self, i: int) -> None:
        """Host columns of world ``i`` -> device (pos, q, v, w, awake, sleep timer)."""
        w = self.worlds[i]
        n = w.body_count
        b0 = self.offsets[i]
        self.ctx.call('upload_state', b0, n, ptr(w._position, D), ptr(w._orientation, D),
                      ptr(w._linear_velocity, D), ptr(w._angular_velocity, D),
                      ptr(w._awake.view(np.uint8), U8), ptr(w._sleep_timer, D))

    def download_state(self, i: int) -> None:
        """Device -> host columns of world ``i`` (state and AABBs)."""
        w = self.worlds[i]
        n = w.body_count
        b0 = self.offsets[i]
        self.ctx.call('download_state', b0, n, ptr(w._position, D), ptr(w._orientation, D),
                      ptr(w._linear_velocity, D), ptr(w._angular_velocity, D),
                      ptr(w._awake.view(np.uint8), U8), ptr(w._sleep_timer, D),
                      ptr(w._aabb_min, D), ptr(w._aabb_max, D))

    def download_joints(self) -> None:
        """Copy the lazily fixed joint state back onto the constraint objects."""
        J = self.packed.n_joints
        if J == 0:
            return
        la = np.zeros((J, 3)); lb = np.zeros((J, 3)); ln = np.zeros(J); acc = np.zeros(J)
        hla = np.zeros(J, np.uint8); hlb = np.zeros(J, np.uint8); hln = np.zeros(J, np.uint8)
        self.ctx.call('download_joints', ptr(la, D), ptr(lb, D), ptr(hla, U8), ptr(hlb, U8),
                      ptr(ln, D), ptr(hln, U8), ptr(acc, D))
        for wi, world in enumerate(self.worlds):
            j0 = self.joint_offsets[wi]
            for k, c in enumerate(world.joint_constraints):
                j = j0 + k
                kind = joint_kind(c)
                if kind == 'motor':
                    c.accum = float(acc[j])
                elif kind == 'distance':
                    if hln[j]:
                        c.length = float(ln[j])
                else:
                    if hla[j]:
                        c.local_a = la[j].copy()
                    if hlb[j]:
                        c.local_b = lb[j].copy()

    def sync_to_host(self) -> None:
        for i in range(len(self.worlds)):
            self.download_state(i)
        self.download_joints()

    # -- results of the last step ------------------------------------------------
    def counts(self):
        W = len(self.worlds)
        p = np.zeros(W, np.int32); c = np.zeros(W, np.int32)
        self.ctx.call('counts', ptr(p, I), ptr(c, I))
        return p, c

    def pairs(self, i: int) -> np.ndarray:
        """Broadphase pairs of world ``i`` (world-local indices), reference order."""
        p, _ = self.counts()
        out = np.zeros((max(int(p[i]), 1), 2), np.int32)
        n = self.ctx.call('get_pairs', i, ptr(out, I), out.shape[0])
        return out[:n] - self.offsets[i]

    def contact_arrays(self, i: int) -> dict:
        _, c = self.counts()
        K = max(int(c[i]), 1)
        a = np.zeros(K, np.int32); b = np.zeros(K, np.int32)
        pt = np.zeros((K, 3)); nr = np.zeros((K, 3)); dp = np.zeros(K); imp = np.zeros((K, 3))
        n = self.ctx.call('get_contacts', i, ptr(a, I), ptr(b, I), ptr(pt, D), ptr(nr, D),
                          ptr(dp, D), ptr(imp, D), K)
        off = self.offsets[i]
        return dict(a=a[:n] - off, b=b[:n] - off, point=pt[:n], normal=nr[:n], depth=dp[:n],
                    impulse=imp[:n])

    def contacts(self, i: int) -> List[Contact]:
        d = self.contact_arrays(i)
        return [Contact(int(d['a'][k]), int(d['b'][k]), d['point'][k], d['normal'][k],
                        float(d['depth'][k]), float(d['impulse'][k, 0]), d['impulse'][k, 1:].copy())
                for k in range(len(d['a']))]

    def islands(self, i: int) -> np.ndarray:
        """Sleep-island label per body of world ``i`` (-1: not in contact)."""
        n = self.worlds[i].body_count
        lab = np.zeros(max(n, 1), np.int32)
        self.ctx.call('get_islands', i, ptr(lab, I))
        lab = lab[:n]
        return np.where(lab >= 0, lab - self.offsets[i], -1)

    def levels(self) -> np.ndarray:
        """Critical path of each world's last contact sweep, in contact solves
        (a wide world: -1 when a thread-block cluster swept it, -2 when the
        many-block sweep did; neither tracks it)."""
        out = np.zeros(len(self.worlds), np.int32)
        self.ctx.call('world_levels', ptr(out, I))
        return out

    def set_cache(self, i: int, a, b, point, impulse) -> None:
        off = self.offsets[i]
        a = np.ascontiguousarray(np.asarray(a, np.int32) + off)
        b = np.ascontiguousarray(np.asarray(b, np.int32) + off)
        point = np.ascontiguousarray(point, 'd').reshape(-1, 3)
        impulse = np.ascontiguousarray(impulse, 'd').reshape(-1, 3)
        self.ctx.call('set_cache', i, len(a), ptr(a, I), ptr(b, I), ptr(point, D), ptr(impulse, D))

    def cache(self, i: int) -> dict:
        cap = 1 << 16
        while True:
            a = np.zeros(cap, np.int32); b = np.zeros(cap, np.int32)
            pt = np.zeros((cap, 3)); imp = np.zeros((cap, 3))
            rc = self.ctx.lib.omi_get_cache(self.ctx.h, i, ptr(a, I), ptr(b, I), ptr(pt, D),
                                            ptr(imp, D), cap)
            if rc == -2 and cap < (1 << 26):
                cap *= 8
                continue
            n = self.ctx.check(rc, 'omi_get_cache')
            off = self.offsets[i]
            return dict(a=a[:n] - off, b=b[:n] - off, point=pt[:n], impulse=imp[:n])

    # -- snapshot / restore ------------------------------------------------------
    def snapshot(self, i: int) -> dict:
        """World ``i``'s resident state and warm-start cache, as host arrays.

        Restoring it (here or into another batch holding the same world) and
        stepping gives exactly what stepping on from here would: pose,
        velocities, sleep state, the solver's warm-start impulses
        (solver.py:91, 272-278) and the sensor overlaps the next step's
        events are formed against are all the step carries over.
        """
        w = self.worlds[i]
        n = w.body_count
        self.download_state(i)
        snap = {'overlaps': set(self.overlaps[i])}
        snap.update({name: np.array(getattr(w, '_' + name)[:n], copy=True)
                     for name in ('position', 'orientation', 'linear_velocity', 'angular_velocity',
                                  'awake', 'sleep_timer')})
        snap['cache'] = self.cache(i)
        snap['time'] = w.time
        return snap

    def restore(self, i: int, snap: dict) -> None:
        """Put a :meth:`snapshot` back into world ``i`` (host columns and device)."""
        w = self.worlds[i]
        n = w.body_count
        for name in ('position', 'orientation', 'linear_velocity', 'angular_velocity', 'awake',
                     'sleep_timer'):
            getattr(w, '_' + name)[:n] = snap[name]
        w.time = snap['time']
        self.overlaps[i] = set(snap.get('overlaps', ()))
        self.upload_state(i)
        c = snap['cache']
        self.set_cache(i, c['a'], c['b'], c['point'], c['impulse'])

    def profile(self) -> dict:
        """Per-stage device milliseconds of one eagerly launched step."""
        return self.ctx.profile_step()
