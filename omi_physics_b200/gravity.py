"""Gravity volumes (``OMI_physics_gravity`` zones), as the reference models them.

A volume is a :class:`~omi_physics_b200.model.Gravity` field plus the region
it acts in (``src/omi_physics/gravity.py:15-79``); volumes apply per body in
ascending ``priority`` (``replace`` overrides, ``stop`` zeroes, otherwise
fields add). The CUDA step resolves them inside its integrate-forces kernel;
this module holds the descriptions and packs them into the device table.
The reference's own volume and region objects pack the same way.
"""
from typing import List, Sequence

import numpy as np

from . import model

#: kind word of one packed volume
VOL_POINT = 1            # field pulls toward its centre (else directional)
VOL_REGION_SPHERE = 2    # region bits (<< 1): 0 everywhere, 1 sphere, 2 box
VOL_REGION_BOX = 4
VOL_REPLACE = 8
VOL_STOP = 16


class SphereRegion:
    """Every point within ``radius`` of ``center`` (gravity.py:15-25)."""

    def __init__(self, center, radius: float):
        self.center = np.asarray(center, dtype='d')
        self.radius = float(radius)

    def contains(self, pos) -> bool:
        d = np.asarray(pos, dtype='d') - self.center
        return bool(np.dot(d, d) <= self.radius ** 2)


class BoxRegion:
    """An axis-aligned box around ``center`` with half-extents ``half`` (gravity.py:28-37)."""

    def __init__(self, center, half):
        self.center = np.asarray(center, dtype='d')
        self.half = np.asarray(half, dtype='d')

    def contains(self, pos) -> bool:
        return bool(np.all(np.abs(np.asarray(pos, dtype='d') - self.center) <= self.half))


class InfiniteRegion:
    """All of space (gravity.py:40-45)."""

    def contains(self, pos) -> bool:
        return True


class GravityVolume:
    """A gravity field with a region of influence (gravity.py:51-79)."""

    def __init__(self, field: model.Gravity, region=None):
        self.field = field
        self.region = region or InfiniteRegion()

    @property
    def priority(self) -> int:
        return self.field.priority


def _unit_times(v, g: float) -> np.ndarray:
    """``mathutil.normalize(v) * g`` with numpy's own arithmetic (mathutil.py:21-24)."""
    v = np.asarray(v, dtype='d')
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    return v / np.maximum(n, 1e-12) * g


def pack_volumes(volumes: Sequence) -> dict:
    """Device table rows for ``volumes`` in application order.

    ``kind`` (int32 flags above), ``g`` (field magnitude), ``field`` (a
    directional field's acceleration, computed here exactly as the reference's
    ``field_at`` computes it, or a point field's centre), ``rc`` (region
    centre) and ``rr`` (a sphere region's ``radius ** 2`` in ``rr[0]``, a box
    region's half-extents). Raises ``ValueError`` for a region that is not a
    sphere, a box or all of space.
    """
    ordered: List = sorted(volumes, key=lambda v: v.priority)     # stable, as gravity.py:89
    m = len(ordered)
    kind = np.zeros(m, np.int32)
    g = np.zeros(m)
    field = np.zeros((m, 3))
    rc = np.zeros((m, 3))
    rr = np.zeros((m, 3))
    for k, v in enumerate(ordered):
        f = v.field
        fl = 0
        if f.type == 'point':
            fl |= VOL_POINT
            field[k] = np.asarray(f.center, dtype='d')
        else:
            field[k] = _unit_times(f.direction, f.gravity)
        g[k] = float(f.gravity)
        if f.replace:
            fl |= VOL_REPLACE
        elif f.stop:
            fl |= VOL_STOP
        reg = v.region
        if hasattr(reg, 'radius') and hasattr(reg, 'center'):
            fl |= VOL_REGION_SPHERE
            rc[k] = np.asarray(reg.center, dtype='d')
            rr[k, 0] = float(reg.radius) ** 2
        elif hasattr(reg, 'half') and hasattr(reg, 'center'):
            fl |= VOL_REGION_BOX
            rc[k] = np.asarray(reg.center, dtype='d')
            rr[k] = np.asarray(reg.half, dtype='d')
        elif type(reg).__name__ != 'InfiniteRegion':
            raise ValueError('gravity volume region %r is not a sphere, a box or everywhere'
                             % type(reg).__name__)
        kind[k] = fl
    return dict(kind=kind, g=g, field=field, rc=rc, rr=rr)

