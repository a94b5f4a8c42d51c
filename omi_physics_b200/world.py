"""``PhysicsWorld`` host mirror: the reference's public world API over the
structure-of-arrays state, stepped by the CUDA backend.

The public surface follows ``src/omi_physics/world.py`` (constructor 30-72,
``add_shape``/``add_material``/``add_filter`` 175-193, ``add_body`` 253-299,
mass properties 301-316 and 614-639, ``step`` 410-430, ``advance`` 399-408,
column views 141-167). The column arrays use the reference's private names
(``_position``, ``_orientation`` ...) because the CUDA backend reads and
writes them by those names on either world class, which is what makes it a
drop-in behind the reference's own ``PhysicsWorld(backend=...)`` slot.

There is no CPU step here: ``step`` runs the same stage sequence as the
reference and every stage is executed by :class:`~omi_physics_b200.backend.
CudaBackend`; constructing a world without a usable CUDA library raises.
"""
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

from . import model

_TYPE_INT = {model.STATIC: 0, model.KINEMATIC: 1, model.DYNAMIC: 2}


def inertia_diagonal(shape: Optional[model.Shape], mass: float) -> np.ndarray:
    """Solid-body inertia diagonal about the centre (world.py:614-639)."""
    if shape is None:
        return np.zeros(3)
    t = shape.type
    if t == 'sphere':
        v = 0.4 * mass * shape.radius ** 2
        return np.array([v, v, v])
    if t == 'box':
        x, y, z = shape.size
        k = mass / 12.0
        return k * np.array([y * y + z * z, x * x + z * z, x * x + y * y])
    if t in ('capsule', 'cylinder'):
        r = shape.radiusBottom
        h = shape.height
        ix = mass * (3 * r * r + h * h) / 12.0
        return np.array([ix, 0.5 * mass * r * r, ix])
    if shape.points is not None and len(shape.points):
        ext = shape.points.max(axis=0) - shape.points.min(axis=0)
        x, y, z = ext
        k = mass / 12.0
        return k * np.array([y * y + z * z, x * x + z * z, x * x + y * y])
    return np.zeros(3)


class PhysicsWorld:
    """A rigid-body world: add shapes/materials/filters, then bodies, then step."""

    _VEC = ('position', 'prev_position', 'orientation', 'prev_orientation',
            'linear_velocity', 'angular_velocity', 'inv_inertia', 'aabb_min', 'aabb_max')
    _SCALAR_F = ('inv_mass', 'mass', 'gravity_factor', 'linear_damping',
                 'angular_damping', 'quadratic_drag', 'sleep_timer', 'restitution_pad')
    _SCALAR_I = ('motion_type', 'collider_shape', 'collider_material',
                 'collider_filter', 'trigger_shape', 'island')

    def __init__(self, gravity: Optional[model.Gravity] = None,
                 fixed_dt: float = 1.0 / 60.0, max_frame: float = 0.25,
                 backend: Any = None, sleep_enabled: bool = True,
                 default_linear_damping: float = 0.0,
                 default_angular_damping: float = 0.0,
                 gpu_threshold: int = 10000,
                 velocity_iterations: int = 10) -> None:
        self.gravity = gravity if gravity is not None else model.Gravity()
        self.gravity_volumes: List[Any] = []
        self.fixed_dt = fixed_dt
        self.max_frame = max_frame
        self.sleep_enabled = sleep_enabled
        self.default_linear_damping = default_linear_damping
        self.default_angular_damping = default_angular_damping
        self.gpu_threshold = gpu_threshold
        self.shapes: List[model.Shape] = []
        self.materials: List[model.Material] = []
        self.filters: List[model.CollisionFilter] = []
        self.joints: List[model.Joint] = []
        self.joint_attachments: List[Any] = []
        self.pair_friction: Dict[Tuple[int, int], Tuple[float, float]] = {}
        self._n = 0
        self._cap = 0
        self._accumulator = 0.0
        self.time = 0.0
        self.bodies: List[Any] = []
        self._alloc(8)
        self._collision: Any = None
        self._velocity_iterations = velocity_iterations
        self.contacts: List[Any] = []
        self.triggers_overlaps: set = set()
        self.trigger_listeners: List[Any] = []
        self.joint_constraints: List[Any] = []
        self.joint_iterations = 10
        if backend is None or isinstance(backend, str):
            if backend not in (None, 'cuda', 'gpu', 'auto'):
                raise ValueError('omi_physics_b200 worlds step on CUDA only, got %r' % backend)
            from .backend import CudaBackend
            backend = CudaBackend()
        self._backend_mode = 'fixed'
        self.backend = backend

    # -- storage -----------------------------------------------------------
    def _alloc(self, cap: int) -> None:
        """Zeroed columns for ``cap`` bodies (identity orientations, awake)."""
        self._cap = cap
        for name in self._VEC:
            setattr(self, '_' + name, np.zeros((cap, 4 if 'orientation' in name else 3)))
        for name in self._SCALAR_F:
            setattr(self, '_' + name, np.zeros(cap))
        for name in self._SCALAR_I:
            setattr(self, '_' + name, np.full(cap, -1, dtype='i4'))
        self._awake = np.ones(cap, dtype=bool)
        self._orientation[:, 3] = 1.0
        self._prev_orientation[:, 3] = 1.0

    def _grow(self) -> None:
        """Double the capacity, keeping every live row."""
        old, new = self._cap, max(8, self._cap * 2)
        for name in self._VEC + self._SCALAR_F + self._SCALAR_I + ('awake',):
            arr = getattr(self, '_' + name)
            out = np.zeros((new,) + arr.shape[1:], dtype=arr.dtype)
            if name in self._SCALAR_I:
                out.fill(-1)
            out[:old] = arr
            setattr(self, '_' + name, out)
        self._orientation[old:, 3] = 1.0
        self._prev_orientation[old:, 3] = 1.0
        self._awake[old:] = True
        self._cap = new

    def _view(self, name: str) -> np.ndarray:
        return getattr(self, '_' + name)[:self._n]

    position = property(lambda s: s._view('position'))
    prev_position = property(lambda s: s._view('prev_position'))
    orientation = property(lambda s: s._view('orientation'))
    prev_orientation = property(lambda s: s._view('prev_orientation'))
    linear_velocity = property(lambda s: s._view('linear_velocity'))
    angular_velocity = property(lambda s: s._view('angular_velocity'))
    inv_mass = property(lambda s: s._view('inv_mass'))
    mass = property(lambda s: s._view('mass'))
    inv_inertia = property(lambda s: s._view('inv_inertia'))
    gravity_factor = property(lambda s: s._view('gravity_factor'))
    linear_damping = property(lambda s: s._view('linear_damping'))
    angular_damping = property(lambda s: s._view('angular_damping'))
    quadratic_drag = property(lambda s: s._view('quadratic_drag'))
    motion_type = property(lambda s: s._view('motion_type'))
    collider_shape = property(lambda s: s._view('collider_shape'))
    collider_material = property(lambda s: s._view('collider_material'))
    collider_filter = property(lambda s: s._view('collider_filter'))
    trigger_shape = property(lambda s: s._view('trigger_shape'))
    aabb_min = property(lambda s: s._view('aabb_min'))
    aabb_max = property(lambda s: s._view('aabb_max'))
    awake = property(lambda s: s._view('awake'))
    island = property(lambda s: s._view('island'))
    sleep_timer = property(lambda s: s._view('sleep_timer'))

    @property
    def body_count(self) -> int:
        """Number of live bodies."""
        return self._n

    # -- document tables ---------------------------------------------------
    def add_shape(self, shape: model.Shape) -> int:
        """Register a shape; return its index."""
        self.shapes.append(shape)
        return len(self.shapes) - 1

    def add_material(self, mat: model.Material) -> int:
        """Register a material; return its index."""
        self.materials.append(mat)
        return len(self.materials) - 1

    def add_filter(self, filt: model.CollisionFilter) -> int:
        """Register a collision filter; return its index."""
        self.filters.append(filt)
        return len(self.filters) - 1

    def add_joint(self, joint: model.Joint) -> int:
        """Register a joint definition (document table only); return its index."""
        self.joints.append(joint)
        return len(self.joints) - 1

    def material_for(self, index: int) -> model.Material:
        """Material at ``index`` or the default one when out of range."""
        if 0 <= index < len(self.materials):
            return self.materials[index]
        return model.DEFAULT_MATERIAL

    def filter_for(self, index: int) -> model.CollisionFilter:
        """Filter at ``index`` or the default one when out of range."""
        if 0 <= index < len(self.filters):
            return self.filters[index]
        return model.DEFAULT_FILTER

    def set_pair_friction(self, material_a: int, material_b: int,
                          static_mu: float, dynamic_mu: float) -> None:
        """Override the friction of one unordered material pair."""
        key = (material_a, material_b) if material_a <= material_b else (material_b, material_a)
        self.pair_friction[key] = (float(static_mu), float(dynamic_mu))

    def pair_friction_for(self, material_a: int, material_b: int):
        """``(static_mu, dynamic_mu)`` override for the pair, or ``None``."""
        key = (material_a, material_b) if material_a <= material_b else (material_b, material_a)
        return self.pair_friction.get(key)

    # -- impulses ----------------------------------------------------------
    def apply_impulse(self, i: int, impulse) -> None:
        """``v += J / m`` on body ``i`` and wake it (world.py:231-238)."""
        self._linear_velocity[i] += self._inv_mass[i] * np.asarray(impulse, dtype='d')
        self.wake(i)

    def apply_angular_impulse(self, i: int, impulse) -> None:
        """``w += I_world^-1 L`` on body ``i`` and wake it (world.py:240-250)."""
        q = self._orientation[i] / max(np.linalg.norm(self._orientation[i]), 1e-12)
        x, y, z, w = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        inv_world = (R * self._inv_inertia[i]) @ R.T
        self._angular_velocity[i] += inv_world @ np.asarray(impulse, dtype='d')
        self.wake(i)

    # -- bodies ------------------------------------------------------------
    def add_body(self, motion: Optional[model.Motion] = None,
                 collider: Optional[model.Collider] = None,
                 trigger: Optional[model.Trigger] = None,
                 position=(0, 0, 0), orientation=(0, 0, 0, 1), handle: Any = None) -> int:
        """Create one body row from its motion/collider; return its index."""
        motion = motion if motion is not None else model.Motion()
        if self._n >= self._cap:
            self._grow()
        i = self._n
        self._n += 1
        self._position[i] = position
        self._prev_position[i] = position
        self._orientation[i] = orientation
        self._prev_orientation[i] = orientation
        self._linear_velocity[i] = motion.linearVelocity
        self._angular_velocity[i] = motion.angularVelocity
        self._motion_type[i] = _TYPE_INT[motion.type]
        self._gravity_factor[i] = motion.gravityFactor
        self._linear_damping[i] = motion.linearDamping
        self._angular_damping[i] = motion.angularDamping
        self._quadratic_drag[i] = motion.quadraticDrag
        self._awake[i] = True
        self._sleep_timer[i] = 0.0
        shape = None
        if collider is not None and 0 <= collider.shape < len(self.shapes):
            shape = self.shapes[collider.shape]
            self._collider_shape[i] = collider.shape
            self._collider_material[i] = collider.physicsMaterial
            self._collider_filter[i] = collider.collisionFilter
            self._collision = self._collision or _DeviceCollisionStub(self._velocity_iterations)
        if trigger is not None and 0 <= trigger.shape < len(self.shapes):
            self._trigger_shape[i] = trigger.shape
            self._collision = self._collision or _DeviceCollisionStub(self._velocity_iterations)
        self._set_mass_properties(i, motion, shape)
        self.bodies.append(handle)
        return i

    def _set_mass_properties(self, i: int, motion: model.Motion, shape) -> None:
        """Mass, inverse mass and inverse inertia diagonal (world.py:301-316)."""
        if motion.type != model.DYNAMIC:
            self._inv_mass[i] = 0.0
            self._mass[i] = 0.0
            self._inv_inertia[i] = 0.0
            return
        m = max(motion.mass, 1e-9)
        self._mass[i] = m
        self._inv_mass[i] = 1.0 / m
        diag = np.asarray(motion.inertiaDiagonal, dtype='d')
        if not diag.any():
            diag = inertia_diagonal(shape, m) if shape is not None else np.zeros(3)
        with np.errstate(divide='ignore'):
            self._inv_inertia[i] = np.where(diag > 0, 1.0 / np.maximum(diag, 1e-12), 0.0)

    # -- masks, gravity ----------------------------------------------------
    def dynamic_mask(self) -> np.ndarray:
        """Awake dynamic bodies."""
        return (self.motion_type == 2) & self.awake

    def moving_mask(self) -> np.ndarray:
        """Awake dynamic or kinematic bodies."""
        return ((self.motion_type == 2) | (self.motion_type == 1)) & self.awake

    def is_awake_mover(self, i: int) -> bool:
        """Awake dynamic body or any kinematic body."""
        t = self._motion_type[i]
        return bool((t == 2 and self._awake[i]) or t == 1)

    def resolve_gravity(self) -> np.ndarray:
        """Per-body gravity ``(N, 3)`` (world.py:386-396); volumes are rejected."""
        base = np.asarray(self.gravity.direction, dtype='d')
        norm = np.linalg.norm(base)
        base = base / norm if norm else base
        return np.tile(base * self.gravity.gravity, (self._n, 1))

    # -- the step ----------------------------------------------------------
    def advance(self, real_dt: float) -> float:
        """Fixed-step accumulator; returns the render interpolation alpha."""
        self._accumulator = min(self._accumulator + real_dt, self.max_frame)
        while self._accumulator >= self.fixed_dt:
            self.step(self.fixed_dt)
            self._accumulator -= self.fixed_dt
        return self._accumulator / self.fixed_dt

    def step(self, dt: float) -> None:
        """One fixed step, in the reference's stage order (world.py:410-430)."""
        self._prev_position[:self._n] = self.position
        self._prev_orientation[:self._n] = self.orientation
        self.backend.integrate_forces(self, dt)
        if self._collision is not None:
            self.backend.refit_aabbs(self)
            self._collision.run(self, dt)
        if self.joint_constraints:
            self._solve_joints(dt)
        self.backend.integrate_positions(self, dt)
        if self.sleep_enabled:
            self._update_sleep(dt)
        self.time += dt

    def _solve_joints(self, dt: float) -> None:
        raise RuntimeError('joints are solved by the CUDA backend; attach it first')

    def _update_sleep(self, dt: float) -> None:
        raise RuntimeError('sleeping is computed by the CUDA backend; attach it first')

    def writeback(self, alpha: float = 1.0):
        """Interpolated render poses (world.py:432-437)."""
        pos = self.prev_position * (1 - alpha) + self.position * alpha
        quat = self.prev_orientation * (1 - alpha) + self.orientation * alpha
        n = np.linalg.norm(quat, axis=-1, keepdims=True)
        return pos, quat / np.maximum(n, 1e-12)

    def wake(self, i: int) -> None:
        """Wake body ``i`` and reset its sleep timer."""
        self._awake[i] = True
        self._sleep_timer[i] = 0.0

    def add_joint_constraint(self, constraint: Any) -> Any:
        """Register a joint constraint and wake the bodies it touches."""
        self.joint_constraints.append(constraint)
        for i in (getattr(constraint, 'a', None), getattr(constraint, 'b', None),
                  getattr(constraint, 'body', None)):
            if i is not None and i >= 0:
                self.wake(i)
        return constraint

    def add_gravity_volume(self, volume: Any) -> Any:
        """Register a gravity zone (an :class:`omi_physics_b200.gravity.GravityVolume`); return it."""
        self.gravity_volumes.append(volume)
        return volume

    def add_trigger_listener(self, fn: Any) -> None:
        """Register ``fn(event_type, trigger_index, other_index)`` (world.py:580-582)."""
        self.trigger_listeners.append(fn)

    def dispatch_trigger(self, event_type: str, trigger_index: int, other_index: int) -> None:
        """Notify every trigger listener of one overlap event (world.py:584-588)."""
        for fn in self.trigger_listeners:
            fn(event_type, trigger_index, other_index)


class _DeviceCollisionStub:
    """Placeholder for the collision stages until the CUDA backend attaches.

    The reference builds ``_CollisionStages`` on the first collider
    (world.py:292); here the attach step replaces this stub with the device
    stage object, carrying over the requested solver iteration count.
    """

    def __init__(self, velocity_iterations: int) -> None:
        self.velocity_iterations = velocity_iterations
        self.solver = self
        self.contacts: List[Any] = []

    def run(self, world, dt):
        raise RuntimeError('collision runs on the CUDA backend; attach it first')
