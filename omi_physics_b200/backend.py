"""``CudaBackend`` — the drop-in compute backend for ``PhysicsWorld``.

It satisfies the reference's backend duck type (``name``,
``integrate_forces(world, dt)``, ``integrate_positions(world, dt)``,
``refit_aabbs(world)``; src/omi_physics/backend.py:21-53) and plugs into the
reference's own slot: ``PhysicsWorld(backend=CudaBackend())`` takes an object
backend as fixed (world.py:335-338). The reference's ``step`` calls the
collision stages, the joint solve and the sleep update directly on the world
(world.py:419-429), so on first use the backend attaches to the world: it
replaces ``world._collision`` with a device-stage object exposing ``run``,
``contacts``, ``solver`` and ``broadphase``, and rebinds ``_solve_joints`` and
``_update_sleep`` on the instance. The world's numpy columns stay the public
source of truth: each step uploads the mutable state, runs the whole step as
one CUDA graph (integrate, refit, broadphase, narrowphase, contact solve,
joints, integrate positions, sleep) and downloads the result.

There is no CPU fallback: without the built library or a CUDA device the
first step raises.
"""
from typing import Any, Optional

from ._lib import OmiError, UnsupportedFeature
from .arena import check_supported, static_signature


class _LazyContacts:
    """``world.contacts`` of the last step, fetched from the device on first use."""

    def __init__(self, batch, index: int):
        self._batch, self._index, self._items = batch, index, None

    def _get(self):
        if self._items is None:
            self._items = self._batch.contacts(self._index)
        return self._items

    def __len__(self):
        return len(self._get())

    def __iter__(self):
        return iter(self._get())

    def __getitem__(self, k):
        return self._get()[k]

    def __bool__(self):
        return len(self) > 0


class _DevicePairs:
    """``broadphase`` stand-in: the last step's pair list, in the reference's order."""

    def __init__(self, backend: 'CudaBackend'):
        self._backend = backend

    def pairs(self, world) -> list:
        b = self._backend._batch
        return [tuple(map(int, p)) for p in b.pairs(0)] if b is not None else []


class _SensorState:
    """``triggers`` stand-in (triggers.py:17-44): the last step's overlaps."""

    def __init__(self, original: Any):
        self.overlaps = set(getattr(getattr(original, 'triggers', None), 'overlaps', set()))


class DeviceCollisionStages:
    """Replaces ``world._collision`` (world.py:642-676) once the backend attaches.

    ``solver`` keeps the original solver object so iteration counts and
    solver parameters set on it keep their effect; the contacts and the
    warm-start cache live on the device. Sensor overlaps are tested on the
    device after the contact solve, as the reference tests them; ``run``
    dispatches the step's enter / stay / exit events to the world's trigger
    listeners (world.py:674-676), sorted within each kind, once the step's
    state is back on the host.
    """

    def __init__(self, backend: 'CudaBackend', original: Any):
        self.backend = backend
        self.solver = getattr(original, 'solver', original)
        self.broadphase = _DevicePairs(backend)
        self.narrowphase = None
        self.triggers = _SensorState(original)
        self.contacts: Any = []

    def run(self, world, dt: float) -> None:
        """The device already ran this stage inside ``integrate_forces``."""
        self.contacts = world.contacts = self.backend.last_contacts()
        b = self.backend._batch
        if b is None or not (b.has_sensors or self.triggers.overlaps):
            return
        new = b.trigger_overlaps(0)
        old = self.triggers.overlaps
        events = ([('enter',) + p for p in sorted(new - old)] + [('stay',) + p for p in sorted(new & old)] +
                  [('exit',) + p for p in sorted(old - new)])
        self.triggers.overlaps = new
        for ev in events:
            world.dispatch_trigger(*ev)


def _noop(dt: float) -> None:
    return None


class CudaBackend:
    """Runs ``PhysicsWorld.step`` on one B200 through the omi_b200 C ABI."""

    name = 'cuda'

    def __init__(self, device: int = 0):
        self.device = device
        self._batch = None
        self._world = None
        self._sig: Optional[tuple] = None
        self._contacts = None

    # -- attach -------------------------------------------------------------
    def attach(self, world) -> None:
        """Take over the world's collision, joint and sleep stages (idempotent)."""
        if self._world is not None and self._world is not world:
            raise ValueError('a CudaBackend serves one world; create one per world')
        check_supported(world)
        col = world._collision
        if col is not None and not isinstance(col, DeviceCollisionStages):
            world._collision = DeviceCollisionStages(self, col)
        world._solve_joints = _noop
        world._update_sleep = _noop
        self._world = world

    def _ensure_loaded(self, world, dt: float) -> None:
        from .batch import WorldBatch
        sig = static_signature(world)
        if self._batch is None or sig != self._sig:
            # a topology change (a body or table added) reloads the arena; the
            # reference's solver keeps its warm-start cache across it, keyed by
            # body pairs whose indices do not change (solver.py:91, 272-278)
            carry = self._batch.cache(0) if self._batch is not None else None
            ctx = self._batch.ctx if self._batch is not None else None
            self._batch = WorldBatch([world], device=self.device, dts=[dt], ctx=ctx)
            self._sig = sig
            if carry is not None and len(carry['a']):
                self._batch.set_cache(0, carry['a'], carry['b'], carry['point'], carry['impulse'])
        else:
            self._batch.upload_state(0)
        self._batch.dts = [dt]
        self._batch.refresh_params()

    # -- the backend duck type ----------------------------------------------
    def integrate_forces(self, world, dt: float) -> None:
        """Upload, then run the entire step for this world on the device."""
        self.attach(world)
        self._ensure_loaded(world, dt)
        b = self._batch
        b.ctx.call('step', 1)
        b.download_state(0)
        if world.joint_constraints:
            b.download_joints()
        self._contacts = None
        world.contacts = self.last_contacts()

    def refit_aabbs(self, world) -> None:
        """AABBs were refit on the device and downloaded with the state."""
        return None

    def integrate_positions(self, world, dt: float) -> None:
        """Positions were integrated on the device inside the same step."""
        return None

    # -- results --------------------------------------------------------------
    def last_contacts(self):
        if self._contacts is None:
            self._contacts = _LazyContacts(self._batch, 0)
        return self._contacts

    def profile(self) -> dict:
        return self._batch.profile() if self._batch is not None else {}


def select_backend(prefer: str = 'cuda') -> CudaBackend:
    """The backend for ``prefer`` in ``cuda``/``gpu``/``auto``; nothing else exists here."""
    if prefer not in ('cuda', 'gpu', 'auto'):
        raise ValueError('omi_physics_b200 provides only the CUDA backend, not %r' % (prefer,))
    return CudaBackend()


__all__ = ['CudaBackend', 'DeviceCollisionStages', 'select_backend', 'OmiError',
           'UnsupportedFeature']
