"""Capsule against triangles on the GPU, behind the reference's own calls.

The reference answers a capsule against a batch of triangles with its
compiled ``capsule_triangles`` (``_collide_native.pyx:454-574``), reached
through ``collide.capsule_triangle_batch``, ``capsule_triangles`` and
``capsule_mesh_pushes`` (``collide.py:385-462``); a character controller
asks that nine to twelve times a frame per character. The functions here
keep those names, arguments and return values — ``(hit, points, normals,
depths)`` lined up with the triangles, normals pointing from the triangle
toward the capsule, zeros where ``hit`` is false — and compute on the device
through the C ABI (``omi_capsule_triangles*``), bit-identical to the
reference. ``capsule_triangles_many`` answers many capsules' candidate sets
in one call, which is the form that fills a GPU: every character of a frame
at once.

A capsule is any object with ``p0``, ``p1`` (segment ends) and ``radius``:
the reference's ``body.CapsuleProxy`` or :class:`CapsuleProxy` below.
"""
import threading
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from ._lib import D, I64, U8, Context, ptr

_CTX: Dict[int, Context] = {}
_LOCK: Dict[int, threading.Lock] = {}
_GUARD = threading.Lock()


def context(device: int = 0) -> Tuple[Context, threading.Lock]:
    """The shared library context of ``device`` and the lock serialising it."""
    with _GUARD:
        if device not in _CTX:
            _CTX[device] = Context(device)
            _LOCK[device] = threading.Lock()
        return _CTX[device], _LOCK[device]


class CapsuleProxy:
    """Segment along the local Y axis plus radius (body.py:80-108)."""
    kind = 'capsule'

    def __init__(self, center, half_height: float, radius: float, rotation):
        self.center = np.asarray(center, dtype='d')
        self.half_height = float(half_height)
        self.radius = float(radius)
        self.R = np.asarray(rotation, dtype='d')
        axis = self.R @ np.array([0.0, 1.0, 0.0])
        self.p0 = self.center - axis * self.half_height
        self.p1 = self.center + axis * self.half_height

    def aabb(self):
        """Axis-aligned bounding box as ``(lo, hi)``."""
        return np.minimum(self.p0, self.p1) - self.radius, np.maximum(self.p0, self.p1) + self.radius


def _outputs(n: int):
    return (np.zeros(n, np.uint8), np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n))


def capsule_triangle_batch(cap, verts, device: int = 0):
    """``collide.capsule_triangle_batch`` (collide.py:438-462): ``verts`` is
    ``(N, 3, 3)``; returns ``(hit (N,) bool, points (N,3), normals (N,3),
    depths (N,))``."""
    verts = np.ascontiguousarray(verts, dtype='d').reshape(-1, 3, 3)
    n = len(verts)
    hit, points, normals, depths = _outputs(n)
    if n:
        p0 = np.ascontiguousarray(cap.p0, dtype='d')
        p1 = np.ascontiguousarray(cap.p1, dtype='d')
        ctx, lock = context(device)
        with lock:
            ctx.call('capsule_triangles', ptr(p0, D), ptr(p1, D), float(cap.radius), ptr(verts, D), n,
                     ptr(hit, U8), ptr(points, D), ptr(normals, D), ptr(depths, D))
    return hit.astype(bool), points, normals, depths


def capsule_triangles(cap, v0, v1, v2, device: int = 0):
    """``collide.capsule_triangles`` (collide.py:385-401): the triangles as
    three ``(N, 3)`` vertex arrays."""
    v0 = np.ascontiguousarray(v0, dtype='d').reshape(-1, 3)
    verts = np.empty((len(v0), 3, 3))
    verts[:, 0] = v0
    verts[:, 1] = np.asarray(v1, dtype='d').reshape(-1, 3)
    verts[:, 2] = np.asarray(v2, dtype='d').reshape(-1, 3)
    return capsule_triangle_batch(cap, verts, device)


def capsule_mesh_pushes(cap, mesh, verts: Optional[np.ndarray] = None, device: int = 0):
    """``collide.capsule_mesh_pushes`` (collide.py:404-435): unit pushes from
    the mesh into the capsule and their depths, deepest first. ``mesh`` is the
    reference's ``TriangleMeshProxy`` (any object with
    ``candidate_vertices(lo, hi)``) unless ``verts`` is given."""
    if verts is None:
        verts = mesh.candidate_vertices(*cap.aabb())
    hit, _points, normals, depths = capsule_triangle_batch(cap, verts, device)
    where = np.flatnonzero(hit)
    if not len(where):
        return np.zeros((0, 3), dtype='d'), np.zeros(0, dtype='d')
    pushes, found = normals[where], depths[where]
    order = np.argsort(-found, kind='stable')
    return pushes[order], found[order]


def pack_capsules(capsules: Sequence) -> np.ndarray:
    """``(q, 7)`` rows ``p0, p1, radius`` of capsule objects."""
    return np.array([np.concatenate([np.asarray(c.p0, 'd'), np.asarray(c.p1, 'd'), [float(c.radius)]])
                     for c in capsules], dtype='d').reshape(-1, 7)


def capsule_triangles_many(caps: np.ndarray, tri_off: np.ndarray, verts: np.ndarray, device: int = 0,
                           out=None):
    """Many capsules at once from host arrays: ``caps`` ``(q, 7)`` (see
    :func:`pack_capsules`), capsule ``c`` owning triangles
    ``tri_off[c]:tri_off[c+1]`` of ``verts`` ``(N, 3, 3)``. Returns
    ``(hit (N,) uint8, points, normals, depths)``; ``out`` may supply those four
    arrays (pinned memory makes the transfers asynchronous)."""
    caps = np.ascontiguousarray(caps, dtype='d').reshape(-1, 7)
    tri_off = np.ascontiguousarray(tri_off, dtype=np.int64)
    verts = np.ascontiguousarray(verts, dtype='d').reshape(-1, 3, 3)
    n = len(verts)
    hit, points, normals, depths = out if out is not None else _outputs(n)
    if n:
        ctx, lock = context(device)
        with lock:
            ctx.call('capsule_triangles_batch', len(caps), ptr(caps, D), ptr(tri_off, I64), ptr(verts, D), n,
                     ptr(hit, U8), ptr(points, D), ptr(normals, D), ptr(depths, D))
    return hit, points, normals, depths


def capsule_triangles_device(ctx: Context, q: int, caps: int, tri_off: int, verts: int, n: int, hit: int,
                             points: int, normals: int, depths: int) -> None:
    """Enqueue the query on ``ctx``'s stream over DEVICE buffers given as raw
    addresses (``tensor.data_ptr()``); returns without waiting."""
    ctx.call('capsule_triangles_device', int(q), int(caps), int(tri_off), int(verts), int(n), int(hit),
             int(points), int(normals), int(depths))


class NativeShim:
    """Stands in for the reference's compiled ``_collide_native`` module
    (``collide._native``): ``capsule_triangles`` runs on the GPU with the
    compiled routine's signature, filling the caller's arrays in place
    (``_collide_native.pyx:454-574``); every other attribute is the wrapped
    module's. Installing it routes the reference's mesh collisions and its
    character controller's depenetration queries through the device::

        from omi_physics import collide
        collide._native = NativeShim(collide._native)
    """

    def __init__(self, native, device: int = 0):
        self._native = native
        self._device = device

    def __getattr__(self, name):
        return getattr(self._native, name)

    def capsule_triangles(self, cp0, cp1, radius, verts, hit, points, normals, depths):
        n = len(verts)
        if not n:
            return
        for a, dt in ((hit, np.uint8), (points, np.float64), (normals, np.float64), (depths, np.float64)):
            if a.dtype != dt or not a.flags['C_CONTIGUOUS']:
                raise ValueError('capsule_triangles writes into C-contiguous %s arrays' % np.dtype(dt).name)
        v = np.ascontiguousarray(verts, dtype='d')
        p0 = np.ascontiguousarray(cp0, dtype='d')
        p1 = np.ascontiguousarray(cp1, dtype='d')
        ctx, lock = context(self._device)
        with lock:
            ctx.call('capsule_triangles', ptr(p0, D), ptr(p1, D), float(radius), ptr(v, D), n, ptr(hit, U8),
                     ptr(points, D), ptr(normals, D), ptr(depths, D))
