"""Joint constraint records solved on the device.

Constructor signatures and attribute names match the reference's
``src/omi_physics/joints.py`` (``PointConstraint`` 60-121,
``DistanceConstraint`` 124-178, ``AngularMotor`` 181-212) so scenes and the
backend treat either set the same way. These classes hold parameters and the
state the reference keeps between steps (lazily fixed local anchors, the rest
length, the motor's accumulated impulse); the arithmetic runs in the CUDA
joint kernel. ``-1`` as a body index means the world.
"""
from typing import Optional

import numpy as np


def _unit(v) -> np.ndarray:
    """``mathutil.normalize`` for one 3-vector: ``v / max(|v|, 1e-12)``."""
    v = np.asarray(v, dtype='d')
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    return v / np.maximum(n, 1e-12)


class PointConstraint:
    """Ball joint holding two anchors coincident (joints.py:60-121)."""
    kind = 'point'

    def __init__(self, a: int, b: int, anchor, local_a: Optional[np.ndarray] = None,
                 local_b: Optional[np.ndarray] = None):
        self.a, self.b = a, b
        self.anchor = np.asarray(anchor, dtype='d')
        self.local_a = local_a
        self.local_b = local_b


class DistanceConstraint:
    """Rigid rod holding ``|pB - pA| == length`` (joints.py:124-178)."""
    kind = 'distance'

    def __init__(self, a: int, b: int, anchor_a, anchor_b, length: Optional[float] = None):
        self.a, self.b = a, b
        self.anchor_a = np.asarray(anchor_a, dtype='d')
        self.anchor_b = np.asarray(anchor_b, dtype='d')
        self.length = length


class AngularMotor:
    """Velocity drive about a world ``axis`` on one body (joints.py:181-212)."""
    kind = 'motor'

    def __init__(self, body: int, axis, target: float, max_force: float = np.inf):
        self.body = body
        self.axis = _unit(axis)
        self.target = float(target)
        self.max_force = max_force
        self.accum = 0.0


def joint_kind(c) -> str:
    """Classify a joint object from either package by its attributes."""
    k = getattr(c, 'kind', None)
    if k in ('point', 'distance', 'motor'):
        return k
    name = type(c).__name__
    if name == 'PointConstraint':
        return 'point'
    if name == 'DistanceConstraint':
        return 'distance'
    if name == 'AngularMotor':
        return 'motor'
    raise TypeError('unsupported joint constraint %r' % (type(c).__name__,))
