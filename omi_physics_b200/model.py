"""OMI physics data model — the input schema of the step.

Field names and defaults are those of the OMI glTF physics extensions, as the
reference defines them in ``src/omi_physics/model.py:33-243``; keeping them
identical is what lets a scene written against the reference load here
unchanged. Only the parts the CUDA step consumes are listed (shapes, motion,
collider, material, collision filter, global gravity) plus the joint/trigger
records so documents round-trip; triangle meshes are taken on static
bodies only (:class:`omi_physics_b200.backend.UnsupportedFeature` otherwise).
"""
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

STATIC = 'static'
KINEMATIC = 'kinematic'
DYNAMIC = 'dynamic'

AVERAGE = 'average'
MINIMUM = 'minimum'
MAXIMUM = 'maximum'
MULTIPLY = 'multiply'

#: combine-mode codes the device tables use
COMBINE_CODES = {AVERAGE: 0, MINIMUM: 1, MAXIMUM: 2, MULTIPLY: 3}


@dataclass
class Shape:
    """``OMI_physics_shape``: one collision proxy, shared by index (model.py:33-82)."""
    type: str = 'box'
    size: tuple = (1.0, 1.0, 1.0)
    radius: float = 0.5
    height: float = 2.0
    radiusBottom: float = 0.5
    radiusTop: float = 0.5
    points: Optional[np.ndarray] = None
    indices: Optional[np.ndarray] = None
    mesh: int = -1

    @classmethod
    def box(cls, size: Sequence[float] = (1.0, 1.0, 1.0)) -> 'Shape':
        """Box with full extents ``size``."""
        return cls(type='box', size=tuple(size))

    @classmethod
    def sphere(cls, radius: float = 0.5) -> 'Shape':
        """Sphere of ``radius``."""
        return cls(type='sphere', radius=float(radius))

    @classmethod
    def convex(cls, points) -> 'Shape':
        """Convex hull of an ``(M, 3)`` local point cloud (its own hull)."""
        return cls(type='convex', points=np.asarray(points, dtype='d'))

    @classmethod
    def trimesh(cls, points, indices) -> 'Shape':
        """Triangle soup: local vertices ``(M, 3)`` and triangles ``(T, 3)``
        (model.py:78-82); collided triangle by triangle, static bodies only."""
        return cls(type='trimesh', points=np.asarray(points, dtype='d'),
                   indices=np.asarray(indices, dtype='i'))

    @classmethod
    def capsule(cls, height: float = 1.0, radius: float = 0.5) -> 'Shape':
        """Capsule: ``height`` is the cylindrical mid-section length."""
        return cls(type='capsule', height=float(height), radiusBottom=float(radius),
                   radiusTop=float(radius))

    @classmethod
    def cylinder(cls, height: float = 2.0, radius: float = 0.5) -> 'Shape':
        """Cylinder of total length ``height``; collided as a capsule of that
        mid-section length, as the reference does (body.py:226-228)."""
        return cls(type='cylinder', height=float(height), radiusBottom=float(radius),
                   radiusTop=float(radius))


@dataclass
class Motion:
    """``OMI_physics_body.motion`` (model.py:86-102)."""
    type: str = DYNAMIC
    mass: float = 1.0
    centerOfMass: tuple = (0.0, 0.0, 0.0)
    inertiaDiagonal: tuple = (0.0, 0.0, 0.0)
    inertiaOrientation: tuple = (0.0, 0.0, 0.0, 1.0)
    linearVelocity: tuple = (0.0, 0.0, 0.0)
    angularVelocity: tuple = (0.0, 0.0, 0.0)
    gravityFactor: float = 1.0
    linearDamping: float = 0.0
    angularDamping: float = 0.0
    quadraticDrag: float = 0.0


@dataclass
class Collider:
    """``OMI_physics_body.collider`` (model.py:106-110)."""
    shape: int = -1
    physicsMaterial: int = -1
    collisionFilter: int = -1


@dataclass
class Trigger:
    """``OMI_physics_body.trigger`` (model.py:113-117): a sensor shape that
    reports overlaps (enter / stay / exit events) and takes no impulse."""
    shape: int = -1
    collisionFilter: int = -1


@dataclass
class Material:
    """A physics material (model.py:121-127)."""
    staticFriction: float = 0.6
    dynamicFriction: float = 0.6
    restitution: float = 0.0
    frictionCombine: str = AVERAGE
    restitutionCombine: str = AVERAGE


@dataclass
class CollisionFilter:
    """Layer/mask filter (model.py:131-155); symmetric ``collides_with``."""
    collisionSystems: tuple = ()
    collideWithSystems: Optional[tuple] = None
    notCollideWithSystems: tuple = ()

    def collides_with(self, other: 'CollisionFilter') -> bool:
        """Both filters must admit each other."""
        return _admits(self, other) and _admits(other, self)


def _admits(a, b) -> bool:
    """``a``'s policy admits a body in ``b``'s systems."""
    theirs = set(b.collisionSystems)
    if theirs & set(a.notCollideWithSystems):
        return False
    if a.collideWithSystems is None:
        return True
    return bool(theirs & set(a.collideWithSystems))


DIRECTIONAL = 'directional'
POINT = 'point'


@dataclass
class Gravity:
    """Global gravity, or the field of a gravity volume (model.py:163-178)."""
    type: str = DIRECTIONAL
    gravity: float = 9.81
    direction: tuple = (0.0, -1.0, 0.0)
    priority: int = 0
    replace: bool = False
    stop: bool = False
    center: tuple = (0.0, 0.0, 0.0)


@dataclass
class JointLimit:
    """One ``OMI_physics_joint`` limit row over a set of axes (model.py:181-189)."""
    linearAxes: tuple = ()
    angularAxes: tuple = ()
    min: float = -np.inf
    max: float = np.inf
    stiffness: float = np.inf
    damping: float = 0.0


@dataclass
class JointDrive:
    """One ``OMI_physics_joint`` drive row (model.py:192-202)."""
    type: str = 'linear'
    mode: str = 'force'
    axis: int = 0
    maxForce: float = np.inf
    positionTarget: Optional[float] = None
    velocityTarget: Optional[float] = None
    stiffness: float = 0.0
    damping: float = 0.0


@dataclass
class Joint:
    """A ``physicsJoints[]`` entry (model.py:205-209); kept for documents only."""
    limits: List = field(default_factory=list)
    drives: List = field(default_factory=list)


@dataclass
class JointAttach:
    """Per-body joint attachment (model.py:212-217); kept for documents only."""
    joint: int = -1
    connectedNode: int = -1
    enableCollision: bool = False


DEFAULT_MATERIAL = Material()
DEFAULT_FILTER = CollisionFilter()


def combine(a: float, b: float, mode: str) -> float:
    """Combine two material coefficients (model.py:231-243)."""
    if mode == MINIMUM:
        return min(a, b)
    if mode == MAXIMUM:
        return max(a, b)
    if mode == MULTIPLY:
        return a * b
    return 0.5 * (a + b)
