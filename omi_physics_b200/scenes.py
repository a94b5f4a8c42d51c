"""Seeded synthetic scenes for the five benchmark workloads.

Every builder takes an ``api`` namespace that provides ``PhysicsWorld``,
``model`` and ``joints`` with the reference's signatures, so the same call
builds an identical scene in this package or in the reference package (the
golden-fixture generator uses the latter). Draw order from
``np.random.default_rng(seed)`` is fixed per builder; a scene is fully
determined by its arguments.

Workloads (sizes and distributions as the benchmark describes them):
  * ``pyramid``      10-level pyramid of 55 unit boxes on a 20x1x20 ground box
  * ``debris``       N bodies, 70% boxes / 30% spheres, density 1000, 40x30x40 m
  * ``convex_pile``  50/25/25 box/sphere/convex in a walled 100x100 m arena
  * ``serving_mix``  request stream of debris worlds, N log-uniform in [16, 2048]
  * ``joint_chain``  pinned chain of 0.2x0.2x1 m links plus loose boxes
  * ``capsule_pile`` capsules / cylinders / boxes / spheres in a walled arena
  * ``zones``        debris through trigger sensors and gravity volumes
  * ``terrain``      capsules, boxes, spheres and hulls on static triangle meshes
  * ``ridge``        one mesh mixing a fine floor with triangles the grid sets aside
  * ``conveyor``     bodies riding a kinematic (sliding, turning) triangle-mesh platform
  * ``degenerate``   coincident centres, zero-depth contacts, sleep and wake-up by a pusher
  * ``rods``         distance joints (world-anchored and body to body) and motors, no point joints
"""
import math
from types import SimpleNamespace
from typing import List, Tuple

import numpy as np


def default_api():
    """This package as a scene-building namespace."""
    from . import gravity, joints, model
    from .world import PhysicsWorld
    return SimpleNamespace(PhysicsWorld=PhysicsWorld, model=model, joints=joints, gravity=gravity)


def _quat_axis_angle(axis: np.ndarray, angle: float) -> Tuple[float, float, float, float]:
    a = axis / np.linalg.norm(axis)
    s = math.sin(0.5 * angle)
    return (float(a[0] * s), float(a[1] * s), float(a[2] * s), float(math.cos(0.5 * angle)))


def _set_iterations(world, iters: int) -> None:
    """Solver iteration count, set where the reference keeps it (world.py:645-654)."""
    world._collision.solver.velocity_iterations = iters


def _new_world(api, backend=None, **kw):
    if backend is not None:
        kw['backend'] = backend
    return api.PhysicsWorld(**kw)


def pyramid(api=None, backend=None, levels: int = 10):
    """Box pyramid: row l has ``levels - l`` unit boxes at y = 0.5 + l."""
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 60.0)
    mat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.5, restitution=0.0))
    ground = w.add_shape(m.Shape.box((20.0, 1.0, 20.0)))
    unit = w.add_shape(m.Shape.box((1.0, 1.0, 1.0)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ground, physicsMaterial=mat),
               position=(0.0, -0.5, 0.0))
    for lvl in range(levels):
        for k in range(levels - lvl):
            x = k - (levels - 1 - lvl) / 2.0
            w.add_body(m.Motion(type=m.DYNAMIC, mass=1.0),
                       m.Collider(shape=unit, physicsMaterial=mat),
                       position=(x, 0.5 + lvl, 0.0))
    _set_iterations(w, 10)
    return w, dict(dt=1.0 / 60.0, steps=120, name='pyramid')


def _debris_into(w, m, n: int, rng, lo=(-20.0, 1.0, -20.0), hi=(20.0, 31.0, 20.0),
                 box_frac: float = 0.7):
    kinds = rng.random(n) < box_frac
    sizes = rng.uniform(0.5, 1.5, size=(n, 3))
    radii = rng.uniform(0.25, 0.75, size=n)
    pos = rng.uniform(lo, hi, size=(n, 3))
    axes = rng.normal(size=(n, 3))
    angles = rng.uniform(0.0, 2.0 * math.pi, size=n)
    mus = rng.uniform(0.3, 0.8, size=n)
    for i in range(n):
        mat = w.add_material(m.Material(staticFriction=float(mus[i]),
                                         dynamicFriction=float(mus[i])))
        if kinds[i]:
            sz = tuple(float(x) for x in sizes[i])
            shape = w.add_shape(m.Shape.box(sz))
            mass = 1000.0 * sz[0] * sz[1] * sz[2]
        else:
            r = float(radii[i])
            shape = w.add_shape(m.Shape.sphere(r))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * r ** 3
        w.add_body(m.Motion(type=m.DYNAMIC, mass=mass),
                   m.Collider(shape=shape, physicsMaterial=mat),
                   position=tuple(float(x) for x in pos[i]),
                   orientation=_quat_axis_angle(axes[i], float(angles[i])))


def debris(api=None, backend=None, n: int = 4096, seed: int = 0, iterations: int = 8,
           extent: float = 20.0, height: float = 30.0, ground: float = 60.0):
    """Random debris field above a static ground box (density 1000 kg/m^3)."""
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0)
    rng = np.random.default_rng(seed)
    gmat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.5))
    gshape = w.add_shape(m.Shape.box((ground, 1.0, ground)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=gshape, physicsMaterial=gmat),
               position=(0.0, -0.5, 0.0))
    _debris_into(w, m, n, rng, lo=(-extent, 1.0, -extent), hi=(extent, 1.0 + height, extent))
    _set_iterations(w, iterations)
    return w, dict(dt=1.0 / 120.0, steps=600, name='debris%d' % n)


def _ellipsoid_points(rng, count: int, semi: np.ndarray) -> np.ndarray:
    d = rng.normal(size=(count, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d * semi


def convex_pile(api=None, backend=None, n: int = 32768, seed: int = 0, iterations: int = 8,
                arena: float = 100.0, height: float = 30.0):
    """Box/sphere/convex pile (50/25/25) in a walled arena; convex via GJK/EPA."""
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0)
    rng = np.random.default_rng(seed)
    gmat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.5))
    floor = w.add_shape(m.Shape.box((arena, 1.0, arena)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=floor, physicsMaterial=gmat),
               position=(0.0, -0.5, 0.0))
    half = arena / 2.0
    wall_x = w.add_shape(m.Shape.box((1.0, 10.0, arena)))
    wall_z = w.add_shape(m.Shape.box((arena, 10.0, 1.0)))
    for sx in (-1.0, 1.0):
        w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=wall_x, physicsMaterial=gmat),
                   position=(sx * (half + 0.5), 5.0, 0.0))
    for sz in (-1.0, 1.0):
        w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=wall_z, physicsMaterial=gmat),
                   position=(0.0, 5.0, sz * (half + 0.5)))
    u = rng.random(n)
    sizes = rng.uniform(0.5, 1.5, size=(n, 3))
    radii = rng.uniform(0.25, 0.75, size=n)
    semis = rng.uniform(0.3, 1.0, size=(n, 3))
    counts = rng.integers(12, 33, size=n)
    lim = half - 2.0
    pos = rng.uniform((-lim, 1.0, -lim), (lim, 1.0 + height, lim), size=(n, 3))
    axes = rng.normal(size=(n, 3))
    angles = rng.uniform(0.0, 2.0 * math.pi, size=n)
    mus = rng.uniform(0.3, 0.8, size=n)
    for i in range(n):
        mat = w.add_material(m.Material(staticFriction=float(mus[i]),
                                         dynamicFriction=float(mus[i])))
        if u[i] < 0.5:
            sz = tuple(float(x) for x in sizes[i])
            shape = w.add_shape(m.Shape.box(sz))
            mass = 1000.0 * sz[0] * sz[1] * sz[2]
        elif u[i] < 0.75:
            r = float(radii[i])
            shape = w.add_shape(m.Shape.sphere(r))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * r ** 3
        else:
            pts = _ellipsoid_points(rng, int(counts[i]), semis[i])
            shape = w.add_shape(m.Shape.convex(pts))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * float(np.prod(semis[i]))
        w.add_body(m.Motion(type=m.DYNAMIC, mass=mass),
                   m.Collider(shape=shape, physicsMaterial=mat),
                   position=tuple(float(x) for x in pos[i]),
                   orientation=_quat_axis_angle(axes[i], float(angles[i])))
    _set_iterations(w, iterations)
    return w, dict(dt=1.0 / 120.0, steps=300, name='convex%d' % n)


def capsule_pile(api=None, backend=None, n: int = 4096, seed: int = 0, iterations: int = 8,
                 arena: float = 40.0, height: float = 20.0):
    """Capsules, cylinders, boxes and spheres (30/20/30/20) in a walled arena.

    Capsule and cylinder pairs go through GJK/EPA (a cylinder is collided as a
    capsule of its length, as the reference does).
    """
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0)
    rng = np.random.default_rng(seed)
    gmat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.5))
    floor = w.add_shape(m.Shape.box((arena, 1.0, arena)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=floor, physicsMaterial=gmat),
               position=(0.0, -0.5, 0.0))
    half = arena / 2.0
    wall_x = w.add_shape(m.Shape.box((1.0, 10.0, arena)))
    wall_z = w.add_shape(m.Shape.box((arena, 10.0, 1.0)))
    for sx in (-1.0, 1.0):
        w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=wall_x, physicsMaterial=gmat),
                   position=(sx * (half + 0.5), 5.0, 0.0))
    for sz in (-1.0, 1.0):
        w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=wall_z, physicsMaterial=gmat),
                   position=(0.0, 5.0, sz * (half + 0.5)))
    u = rng.random(n)
    sizes = rng.uniform(0.5, 1.5, size=(n, 3))
    radii = rng.uniform(0.2, 0.5, size=n)
    lengths = rng.uniform(0.4, 1.6, size=n)
    lim = half - 2.0
    pos = rng.uniform((-lim, 1.0, -lim), (lim, 1.0 + height, lim), size=(n, 3))
    axes = rng.normal(size=(n, 3))
    angles = rng.uniform(0.0, 2.0 * math.pi, size=n)
    mus = rng.uniform(0.3, 0.8, size=n)
    for i in range(n):
        mat = w.add_material(m.Material(staticFriction=float(mus[i]),
                                         dynamicFriction=float(mus[i])))
        r, h = float(radii[i]), float(lengths[i])
        if u[i] < 0.3:
            shape = w.add_shape(m.Shape.capsule(h, r))
            mass = 1000.0 * (math.pi * r * r * h + (4.0 / 3.0) * math.pi * r ** 3)
        elif u[i] < 0.5:
            shape = w.add_shape(m.Shape.cylinder(h, r))
            mass = 1000.0 * math.pi * r * r * h
        elif u[i] < 0.8:
            sz = tuple(float(x) for x in sizes[i])
            shape = w.add_shape(m.Shape.box(sz))
            mass = 1000.0 * sz[0] * sz[1] * sz[2]
        else:
            shape = w.add_shape(m.Shape.sphere(r + 0.1))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * (r + 0.1) ** 3
        w.add_body(m.Motion(type=m.DYNAMIC, mass=mass),
                   m.Collider(shape=shape, physicsMaterial=mat),
                   position=tuple(float(x) for x in pos[i]),
                   orientation=_quat_axis_angle(axes[i], float(angles[i])))
    _set_iterations(w, iterations)
    return w, dict(dt=1.0 / 120.0, steps=300, name='capsules%d' % n)


def zones(api=None, backend=None, n: int = 120, seed: int = 0, iterations: int = 8,
          extent: float = 5.0, height: float = 8.0):
    """Debris falling through trigger sensors and gravity volumes.

    Sensors: a static box zone on the ground, a static sphere zone in the air,
    a kinematic platform carrying a collider and a sensor (its pairs are sensor
    pairs, so it pushes nothing), and a falling dynamic body that is a sensor
    only. Gravity volumes, in priority order: a weak everywhere wind (adds), a
    point attractor in a sphere (adds), a sideways box column (replaces) and a
    zero-gravity box column (stops).
    """
    api = api or default_api()
    m, G = api.model, api.gravity
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0)
    rng = np.random.default_rng(seed)
    gmat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.5))
    ground = w.add_shape(m.Shape.box((4.0 * extent, 1.0, 4.0 * extent)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ground, physicsMaterial=gmat),
               position=(0.0, -0.5, 0.0))
    pad = w.add_shape(m.Shape.box((4.0, 2.0, 4.0)))
    w.add_body(m.Motion(type=m.STATIC), trigger=m.Trigger(shape=pad), position=(3.0, 1.0, 3.0))
    ball = w.add_shape(m.Shape.sphere(2.0))
    w.add_body(m.Motion(type=m.STATIC), trigger=m.Trigger(shape=ball), position=(-3.0, 3.0, -2.0))
    deck = w.add_shape(m.Shape.box((1.5, 0.4, 1.5)))
    halo = w.add_shape(m.Shape.sphere(1.2))
    w.add_body(m.Motion(type=m.KINEMATIC, linearVelocity=(0.6, 0.0, 0.0)),
               m.Collider(shape=deck, physicsMaterial=gmat), trigger=m.Trigger(shape=halo),
               position=(-4.0, 0.5, 3.0))
    probe = w.add_shape(m.Shape.capsule(0.6, 0.3))
    w.add_body(m.Motion(type=m.DYNAMIC, mass=2.0), trigger=m.Trigger(shape=probe),
               position=(0.5, 9.0, 0.5))
    kinds = rng.random(n)
    sizes = rng.uniform(0.4, 1.0, size=(n, 3))
    radii = rng.uniform(0.2, 0.5, size=n)
    pos = rng.uniform((-extent, 1.0, -extent), (extent, 1.0 + height, extent), size=(n, 3))
    axes = rng.normal(size=(n, 3))
    angles = rng.uniform(0.0, 2.0 * math.pi, size=n)
    for i in range(n):
        if kinds[i] < 0.5:
            sz = tuple(float(x) for x in sizes[i])
            shape = w.add_shape(m.Shape.box(sz))
            mass = 1000.0 * sz[0] * sz[1] * sz[2]
        elif kinds[i] < 0.8:
            r = float(radii[i])
            shape = w.add_shape(m.Shape.sphere(r))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * r ** 3
        else:
            r, h = float(radii[i]), float(sizes[i, 0])
            shape = w.add_shape(m.Shape.capsule(h, r))
            mass = 1000.0 * (math.pi * r * r * h + (4.0 / 3.0) * math.pi * r ** 3)
        w.add_body(m.Motion(type=m.DYNAMIC, mass=mass), m.Collider(shape=shape, physicsMaterial=gmat),
                   position=tuple(float(x) for x in pos[i]),
                   orientation=_quat_axis_angle(axes[i], float(angles[i])))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(gravity=0.5, direction=(0.0, 0.0, 1.0), priority=0)))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(type='point', gravity=6.0, center=(0.0, 4.0, 0.0),
                                                   priority=1), G.SphereRegion((0.0, 4.0, 0.0), 3.0)))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(gravity=4.0, direction=(1.0, 0.2, 0.0), priority=2,
                                                   replace=True),
                                         G.BoxRegion((-3.0, 5.0, 3.0), (1.5, 5.0, 1.5))))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(priority=3, stop=True),
                                         G.BoxRegion((3.0, 6.0, -3.0), (1.5, 6.0, 1.5))))
    _set_iterations(w, iterations)
    return w, dict(dt=1.0 / 120.0, steps=300, name='zones%d' % n)


def _grid_mesh(cells: int, extent: float, amp: float, phase: float):
    """A rippled square grid in the xz plane: vertices ``(cells+1)^2``, two
    triangles per cell."""
    xs = np.linspace(-extent, extent, cells + 1)
    pts = np.array([(x, amp * math.sin(0.9 * i + phase) * math.cos(0.7 * j), z)
                    for i, x in enumerate(xs) for j, z in enumerate(xs)], dtype='d')
    idx = []
    for i in range(cells):
        for j in range(cells):
            a, b = i * (cells + 1) + j, (i + 1) * (cells + 1) + j
            idx.append((a, b, a + 1))
            idx.append((b, b + 1, a + 1))
    return pts, np.array(idx, dtype=np.int64)


def terrain(api=None, backend=None, n: int = 60, seed: int = 0, iterations: int = 8,
            cells: int = 24, extent: float = 6.0):
    """Bodies falling onto static triangle meshes: a rippled floor large
    enough for the reference's triangle grid and a small tilted ramp it scans
    exactly. 40% capsules (the batched capsule route), the rest boxes,
    spheres and hulls (GJK/EPA against each candidate triangle)."""
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0)
    rng = np.random.default_rng(seed)
    gmat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.5))
    pts, idx = _grid_mesh(cells, extent, 0.15, 0.3)
    floor = w.add_shape(m.Shape.trimesh(pts, idx))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=floor, physicsMaterial=gmat), position=(0.0, 0.0, 0.0))
    rp, ri = _grid_mesh(4, 1.5, 0.0, 0.0)
    ramp = w.add_shape(m.Shape.trimesh(rp, ri))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ramp, physicsMaterial=gmat), position=(2.5, 0.8, -2.0),
               orientation=_quat_axis_angle(np.array([1.0, 0.0, 0.3]), 0.35))
    u = rng.random(n)
    lim = extent - 1.5
    pos = rng.uniform((-lim, 1.0, -lim), (lim, 5.0, lim), size=(n, 3))
    axes = rng.normal(size=(n, 3))
    angles = rng.uniform(0.0, 2.0 * math.pi, size=n)
    for i in range(n):
        r = float(rng.uniform(0.2, 0.4))
        if u[i] < 0.4:
            h = float(rng.uniform(0.3, 0.9))
            shape = w.add_shape(m.Shape.capsule(h, r))
            mass = 1000.0 * (math.pi * r * r * h + (4.0 / 3.0) * math.pi * r ** 3)
        elif u[i] < 0.6:
            sz = tuple(float(x) for x in rng.uniform(0.3, 0.8, 3))
            shape = w.add_shape(m.Shape.box(sz))
            mass = 1000.0 * sz[0] * sz[1] * sz[2]
        elif u[i] < 0.8:
            shape = w.add_shape(m.Shape.sphere(r))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * r ** 3
        else:
            semi = rng.uniform(0.2, 0.5, 3)
            shape = w.add_shape(m.Shape.convex(_ellipsoid_points(rng, 12, semi)))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * float(np.prod(semi))
        w.add_body(m.Motion(type=m.DYNAMIC, mass=mass), m.Collider(shape=shape, physicsMaterial=gmat),
                   position=tuple(float(x) for x in pos[i]),
                   orientation=_quat_axis_angle(axes[i], float(angles[i])))
    _set_iterations(w, iterations)
    return w, dict(dt=1.0 / 120.0, steps=300, name='terrain%d' % n)


def ridge(api=None, backend=None, n: int = 60, seed: int = 0, iterations: int = 8, cells: int = 32,
          extent: float = 8.0):
    """Bodies falling onto one static mesh that holds a fine rippled floor and
    two large sloped triangles across it: the large ones span more than 64
    of the triangle grid's cells, so the grid keeps them aside and hands them
    to every query (trigrid.py:84-97)."""
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0)
    rng = np.random.default_rng(seed)
    gmat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.5))
    pts, idx = _grid_mesh(cells, extent, 0.1, 1.1)
    k = len(pts)
    ramp = np.array([(-extent, 0.2, 1.0), (extent, 0.2, 1.0), (-extent, 2.5, extent), (extent, 2.5, extent)])
    pts = np.concatenate([pts, ramp])
    idx = np.concatenate([idx, np.array([(k, k + 2, k + 1), (k + 1, k + 2, k + 3)], dtype=idx.dtype)])
    mesh = w.add_shape(m.Shape.trimesh(pts, idx))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=mesh, physicsMaterial=gmat), position=(0.0, 0.0, 0.0))
    lim = extent - 1.5
    pos = rng.uniform((-lim, 3.0, -lim), (lim, 7.0, lim), size=(n, 3))
    axes = rng.normal(size=(n, 3))
    angles = rng.uniform(0.0, 2.0 * math.pi, size=n)
    u = rng.random(n)
    for i in range(n):
        r = float(rng.uniform(0.2, 0.4))
        if u[i] < 0.5:
            h = float(rng.uniform(0.3, 0.9))
            shape = w.add_shape(m.Shape.capsule(h, r))
            mass = 1000.0 * (math.pi * r * r * h + (4.0 / 3.0) * math.pi * r ** 3)
        elif u[i] < 0.75:
            sz = tuple(float(x) for x in rng.uniform(0.3, 0.8, 3))
            shape = w.add_shape(m.Shape.box(sz))
            mass = 1000.0 * sz[0] * sz[1] * sz[2]
        else:
            shape = w.add_shape(m.Shape.sphere(r))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * r ** 3
        w.add_body(m.Motion(type=m.DYNAMIC, mass=mass), m.Collider(shape=shape, physicsMaterial=gmat),
                   position=tuple(float(x) for x in pos[i]),
                   orientation=_quat_axis_angle(axes[i], float(angles[i])))
    _set_iterations(w, iterations)
    return w, dict(dt=1.0 / 120.0, steps=300, name='ridge%d' % n)


def conveyor(api=None, backend=None, n: int = 50, seed: int = 0, iterations: int = 8, cells: int = 16,
             extent: float = 5.0):
    """Bodies falling onto a kinematic triangle-mesh platform that slides and
    turns (its mesh proxy and grid rebuilt every step, as the reference does)
    above a static ground box."""
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0)
    rng = np.random.default_rng(seed)
    gmat = w.add_material(m.Material(staticFriction=0.6, dynamicFriction=0.6))
    ground = w.add_shape(m.Shape.box((8.0 * extent, 1.0, 8.0 * extent)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ground, physicsMaterial=gmat), position=(0.0, -3.5, 0.0))
    pts, idx = _grid_mesh(cells, extent, 0.12, 0.7)
    deck = w.add_shape(m.Shape.trimesh(pts, idx))
    w.add_body(m.Motion(type=m.KINEMATIC, linearVelocity=(0.4, 0.0, 0.1), angularVelocity=(0.0, 0.25, 0.0)),
               m.Collider(shape=deck, physicsMaterial=gmat), position=(0.0, 0.0, 0.0))
    lim = extent - 1.0
    pos = rng.uniform((-lim, 1.0, -lim), (lim, 4.0, lim), size=(n, 3))
    axes = rng.normal(size=(n, 3))
    angles = rng.uniform(0.0, 2.0 * math.pi, size=n)
    u = rng.random(n)
    for i in range(n):
        r = float(rng.uniform(0.2, 0.4))
        if u[i] < 0.4:
            h = float(rng.uniform(0.3, 0.8))
            shape = w.add_shape(m.Shape.capsule(h, r))
            mass = 1000.0 * (math.pi * r * r * h + (4.0 / 3.0) * math.pi * r ** 3)
        elif u[i] < 0.7:
            sz = tuple(float(x) for x in rng.uniform(0.3, 0.7, 3))
            shape = w.add_shape(m.Shape.box(sz))
            mass = 1000.0 * sz[0] * sz[1] * sz[2]
        elif u[i] < 0.85:
            shape = w.add_shape(m.Shape.sphere(r))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * r ** 3
        else:
            semi = rng.uniform(0.2, 0.45, 3)
            shape = w.add_shape(m.Shape.convex(_ellipsoid_points(rng, 12, semi)))
            mass = 1000.0 * (4.0 / 3.0) * math.pi * float(np.prod(semi))
        w.add_body(m.Motion(type=m.DYNAMIC, mass=mass), m.Collider(shape=shape, physicsMaterial=gmat),
                   position=tuple(float(x) for x in pos[i]),
                   orientation=_quat_axis_angle(axes[i], float(angles[i])))
    _set_iterations(w, iterations)
    return w, dict(dt=1.0 / 120.0, steps=300, name='conveyor%d' % n)


def joint_chain(api=None, backend=None, links: int = 32, loose: int = 128, seed: int = 0,
                motor_frac: float = 0.1, iterations: int = 12):
    """Chain of 0.2x0.2x1 m links pinned to the world at both ends, loose boxes above.

    Links share the collision system ``'link'`` and ignore each other, so the
    only link-link coupling is the point joints; loose boxes and the ground
    use the default filter and collide with everything.
    """
    api = api or default_api()
    m, J = api.model, api.joints
    w = _new_world(api, backend, fixed_dt=1.0 / 240.0)
    rng = np.random.default_rng(seed)
    gmat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.5))
    link_filter = w.add_filter(m.CollisionFilter(collisionSystems=('link',),
                                                 notCollideWithSystems=('link',)))
    ground = w.add_shape(m.Shape.box((4.0 * links, 1.0, 40.0)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ground, physicsMaterial=gmat),
               position=(0.0, -0.5, 0.0))
    link_shape = w.add_shape(m.Shape.box((1.0, 0.2, 0.2)))
    y = 3.0
    x0 = -links / 2.0
    first = w.body_count
    for i in range(links):
        w.add_body(m.Motion(type=m.DYNAMIC, mass=2.0),
                   m.Collider(shape=link_shape, physicsMaterial=gmat, collisionFilter=link_filter),
                   position=(x0 + i + 0.5, y, 0.0))
    motor_axes = rng.normal(size=(links + 1, 3))
    motor_on = rng.random(links + 1) < motor_frac
    for i in range(links + 1):
        a = first + i - 1 if i > 0 else -1
        b = first + i if i < links else -1
        w.add_joint_constraint(J.PointConstraint(a, b, (x0 + i, y, 0.0)))
        if motor_on[i]:
            body = b if b >= 0 else a
            w.add_joint_constraint(J.AngularMotor(body, motor_axes[i], 1.0, max_force=50.0))
    sizes = rng.uniform(0.3, 0.6, size=(loose, 3))
    pos = rng.uniform((x0, 4.0, -1.0), (-x0, 12.0, 1.0), size=(loose, 3))
    axes = rng.normal(size=(loose, 3))
    angles = rng.uniform(0.0, 2.0 * math.pi, size=loose)
    bshape_cache = {}
    for i in range(loose):
        sz = tuple(float(x) for x in sizes[i])
        shape = w.add_shape(m.Shape.box(sz))
        bshape_cache[i] = shape
        w.add_body(m.Motion(type=m.DYNAMIC, mass=1000.0 * sz[0] * sz[1] * sz[2]),
                   m.Collider(shape=shape, physicsMaterial=gmat),
                   position=tuple(float(x) for x in pos[i]),
                   orientation=_quat_axis_angle(axes[i], float(angles[i])))
    _set_iterations(w, iterations)
    w.joint_iterations = iterations
    return w, dict(dt=1.0 / 240.0, steps=480, name='chain%d' % links)


def feature_mix(api=None, backend=None, n: int = 70, seed: int = 11):
    """Sphere/box mix exercising restitution, every combine mode, a pair-friction
    override, collision filters, a kinematic mover and a body without collider."""
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0, default_linear_damping=0.05)
    rng = np.random.default_rng(seed)
    g = w.add_material(m.Material(dynamicFriction=0.4, restitution=0.3))
    bouncy = w.add_material(m.Material(dynamicFriction=0.9, restitution=0.8,
                                       frictionCombine=m.MINIMUM, restitutionCombine=m.MAXIMUM))
    slick = w.add_material(m.Material(dynamicFriction=0.1, frictionCombine=m.MULTIPLY))
    w.set_pair_friction(g, slick, 0.7, 0.65)
    f_a = w.add_filter(m.CollisionFilter(collisionSystems=('a',), notCollideWithSystems=('b',)))
    f_b = w.add_filter(m.CollisionFilter(collisionSystems=('b',)))
    ground = w.add_shape(m.Shape.box((16.0, 1.0, 16.0)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ground, physicsMaterial=g),
               position=(0.0, -0.5, 0.0))
    kin = w.add_shape(m.Shape.box((2.0, 0.4, 2.0)))
    w.add_body(m.Motion(type=m.KINEMATIC, linearVelocity=(0.3, 0.0, 0.0),
                        angularVelocity=(0.0, 0.5, 0.0)),
               m.Collider(shape=kin, physicsMaterial=g), position=(-2.0, 0.2, 0.0))
    mats = (g, bouncy, slick, -1)
    for i in range(n):
        r = float(rng.uniform(0.2, 0.5))
        sh = w.add_shape(m.Shape.sphere(r) if i % 3 else
                         m.Shape.box(tuple(float(x) for x in rng.uniform(0.3, 0.8, 3))))
        filt = (-1, f_a, f_b)[i % 3]
        w.add_body(m.Motion(type=m.DYNAMIC, mass=float(rng.uniform(0.5, 3.0)),
                            linearVelocity=tuple(float(x) for x in rng.normal(0, 1.0, 3)),
                            linearDamping=float(rng.uniform(0, 0.2)),
                            angularDamping=float(rng.uniform(0, 0.2)),
                            quadraticDrag=float(rng.uniform(0, 0.05)),
                            gravityFactor=float(rng.uniform(0.5, 1.5))),
                   m.Collider(shape=sh, physicsMaterial=mats[i % 4], collisionFilter=filt),
                   position=tuple(float(x) for x in rng.uniform((-4, 0.5, -4), (4, 6, 4))))
    w.add_body(m.Motion(type=m.DYNAMIC), None, position=(9.0, 3.0, 0.0))
    _set_iterations(w, 6)
    return w, dict(dt=1.0 / 120.0, steps=120, name='feature_mix')


def degenerate(api=None, backend=None):
    """Edge cases of the contact routes and the sleep logic in one world.

    Coincident centres (box-box, sphere-sphere, a sphere inside a box), contacts
    of exactly zero depth (a sphere on a box top, a box stack face to face, a
    capsule lying on the ground), an off-centre mass with an explicit rotated
    inertia, a body far from everything else, and a row of boxes at rest that
    falls asleep before a kinematic pusher reaches and wakes it.
    """
    api = api or default_api()
    m = api.model
    w = _new_world(api, backend, fixed_dt=1.0 / 60.0)
    mat = w.add_material(m.Material(staticFriction=0.6, dynamicFriction=0.5, restitution=0.0))
    ground = w.add_shape(m.Shape.box((40.0, 1.0, 40.0)))
    unit = w.add_shape(m.Shape.box((1.0, 1.0, 1.0)))
    ball = w.add_shape(m.Shape.sphere(0.5))
    small = w.add_shape(m.Shape.sphere(0.3))
    wide = w.add_shape(m.Shape.box((1.5, 1.5, 1.5)))
    pill = w.add_shape(m.Shape.capsule(1.0, 0.25))
    tetra = w.add_shape(m.Shape.convex(np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0],
                                                 [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])))
    pusher = w.add_shape(m.Shape.box((0.5, 1.0, 3.0)))

    def body(shape, pos, q=(0.0, 0.0, 0.0, 1.0), **motion):
        kind = motion.pop('type', m.DYNAMIC)
        return w.add_body(m.Motion(type=kind, **motion),
                          m.Collider(shape=shape, physicsMaterial=mat),
                          position=pos, orientation=q)

    body(ground, (0.0, -0.5, 0.0), type=m.STATIC)
    body(unit, (0.0, 1.5, 0.0))                       # two boxes, one centre
    body(unit, (0.0, 1.5, 0.0))
    body(ball, (3.0, 1.5, 0.0))                       # two spheres, one centre
    body(ball, (3.0, 1.5, 0.0))
    body(wide, (6.0, 1.2, 0.0))                       # a sphere inside a box, same centre
    body(small, (6.0, 1.2, 0.0))
    body(unit, (-3.0, 0.5, 0.0))                      # zero-depth: box on ground, sphere on box
    body(small, (-3.0, 1.3, 0.0))
    body(unit, (-6.0, 0.5, 0.0))                      # face-to-face stack at rest
    body(unit, (-6.0, 1.5, 0.0))
    body(pill, (-9.0, 0.25, 0.0), _quat_axis_angle(np.array([0.0, 0.0, 1.0]), 0.5 * math.pi))
    body(tetra, (-12.0, 0.0, 0.0))                    # hull resting on a face, zero depth
    body(unit, (0.0, 1.0, 4.0), _quat_axis_angle(np.array([0.0, 1.0, 0.0]), 0.25 * math.pi),
         mass=2.0, centerOfMass=(0.2, 0.0, 0.1), inertiaDiagonal=(0.3, 0.5, 0.4),
         inertiaOrientation=_quat_axis_angle(np.array([0.0, 0.0, 1.0]), math.pi / 6.0))
    body(ball, (5000.0, 10.0, -5000.0))               # far from everything
    for k in range(4):                                # a resting row, asleep before the pusher
        body(unit, (8.0 + k, 0.5, 4.0))
    body(pusher, (13.5, 0.5, 4.0), type=m.KINEMATIC, linearVelocity=(-1.0, 0.0, 0.0))
    _set_iterations(w, 8)
    return w, dict(dt=1.0 / 60.0, steps=300, name='degenerate')


def rods(api=None, backend=None, seed: int = 6):
    """Distance joints and motors without point joints (every joint a scalar
    solve): pendulums hung from world anchors, ropes of spheres linked body to
    body with off-centre anchors, one rod given an explicit length, motors on
    some links, and boxes dropping through."""
    api = api or default_api()
    m, J = api.model, api.joints
    w = _new_world(api, backend, fixed_dt=1.0 / 120.0)
    rng = np.random.default_rng(seed)
    mat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.4, restitution=0.1))
    ground = w.add_shape(m.Shape.box((24.0, 1.0, 24.0)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ground, physicsMaterial=mat), position=(0.0, -0.5, 0.0))
    bob = w.add_shape(m.Shape.sphere(0.3))
    link = w.add_shape(m.Shape.box((0.3, 0.8, 0.3)))
    for p in range(4):                                  # pendulums from world anchors
        x = -6.0 + 4.0 * p
        i = w.add_body(m.Motion(type=m.DYNAMIC, mass=1.5), m.Collider(shape=link, physicsMaterial=mat),
                       position=(x + 1.5, 6.0, 0.0), orientation=_quat_axis_angle(np.array([0.0, 0.0, 1.0]), 0.6))
        length = 1.8 if p == 3 else None                # an explicit rest length, else the separation
        w.add_joint_constraint(J.DistanceConstraint(-1, i, (x, 7.0, 0.0), (0.0, 0.4, 0.0), length))
        if p % 2 == 0:
            w.add_joint_constraint(J.AngularMotor(i, tuple(float(v) for v in rng.normal(size=3)), 2.0,
                                                  max_force=20.0))
    for r in range(3):                                  # ropes of spheres, body to body
        z = -4.0 + 4.0 * r
        prev = -1
        for k in range(6):
            i = w.add_body(m.Motion(type=m.DYNAMIC, mass=0.7), m.Collider(shape=bob, physicsMaterial=mat),
                           position=(0.8 * k, 8.0, z))
            anchor_prev = (0.8 * k - 0.8, 8.0, z) if prev < 0 else (0.3, 0.0, 0.0)
            w.add_joint_constraint(J.DistanceConstraint(prev, i, anchor_prev, (-0.3, 0.0, 0.0)))
            prev = i
    for k in range(12):                                 # boxes dropping through
        sz = tuple(float(v) for v in rng.uniform(0.3, 0.7, 3))
        w.add_body(m.Motion(type=m.DYNAMIC, mass=float(rng.uniform(0.5, 2.0))),
                   m.Collider(shape=w.add_shape(m.Shape.box(sz)), physicsMaterial=mat),
                   position=tuple(float(v) for v in rng.uniform((-6.0, 9.0, -5.0), (6.0, 12.0, 5.0))),
                   orientation=_quat_axis_angle(rng.normal(size=3), float(rng.uniform(0, 2 * math.pi))))
    _set_iterations(w, 8)
    w.joint_iterations = 10
    return w, dict(dt=1.0 / 120.0, steps=240, name='rods')


#: the golden-fixture scenes (tests/golden/make_golden.py), by fixture name
GOLDEN_SCENES = {
    'pyramid': lambda api=None, backend=None: pyramid(api, backend),
    'debris': lambda api=None, backend=None: debris(api, backend, n=200, seed=3, extent=6.0,
                                                    height=8.0, ground=20.0),
    'convex': lambda api=None, backend=None: convex_pile(api, backend, n=96, seed=5, arena=8.0,
                                                         height=6.0),
    'chain': lambda api=None, backend=None: joint_chain(api, backend, links=12, loose=16, seed=2),
    'spheres': lambda api=None, backend=None: feature_mix(api, backend),
    'capsules': lambda api=None, backend=None: capsule_pile(api, backend, n=96, seed=7, arena=8.0,
                                                           height=6.0),
    'zones': lambda api=None, backend=None: zones(api, backend),
    'terrain': lambda api=None, backend=None: terrain(api, backend),
    'ridge': lambda api=None, backend=None: ridge(api, backend),
    'conveyor': lambda api=None, backend=None: conveyor(api, backend),
    'degenerate': lambda api=None, backend=None: degenerate(api, backend),
    'rods': lambda api=None, backend=None: rods(api, backend),
    # a hull pile late in its settling, some of it asleep (the convex configuration's regime)
    'convex_late': lambda api=None, backend=None: convex_pile(api, backend, n=1200, seed=13, arena=16.0,
                                                              height=8.0),
}


def serving_requests(n_worlds: int = 1024, seed: int = 0, rate: float = 200.0,
                     n_min: int = 16, n_max: int = 2048) -> List[dict]:
    """The serving request stream: Poisson arrivals, log-uniform world sizes.

    Each request is ``dict(arrival=s, bodies=N, steps=S, seed=k)``; the world
    itself is ``debris(n=N, seed=k)`` scaled to the body count.
    """
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n_worlds)
    arrivals = np.cumsum(gaps)
    sizes = np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=n_worlds)).astype(int)
    steps = rng.integers(60, 601, size=n_worlds)
    return [dict(arrival=float(arrivals[i]), bodies=int(sizes[i]), steps=int(steps[i]),
                 seed=int(seed * 100003 + i)) for i in range(n_worlds)]


def serving_world(req: dict, api=None, backend=None):
    """Debris-style world for one serving request, volume scaled to its size."""
    n = req['bodies']
    ext = max(2.0, 20.0 * (n / 4096.0) ** (1.0 / 3.0))
    return debris(api, backend, n=n, seed=req['seed'], extent=ext, height=1.5 * ext,
                  ground=3.0 * ext)


def joint_chains(n_worlds: int = 512, seed: int = 21, api=None, backend=None, which=None):
    """The batched joints configuration: ``n_worlds`` chains of 16-128 links
    (point joints, 10% with an angular motor) under 64-512 loose boxes,
    1/240 s, 12 contact and 12 joint iterations. Returns ``(worlds, dts)``;
    ``which`` (indices) builds only those worlds of the configuration."""
    rng = np.random.default_rng(seed)
    sizes = [(int(rng.integers(16, 129)), int(rng.integers(64, 513))) for _ in range(n_worlds)]
    worlds, dts = [], []
    for k in (range(n_worlds) if which is None else which):
        w, meta = joint_chain(api, backend, links=sizes[k][0], loose=sizes[k][1], seed=1000 + k)
        worlds.append(w)
        dts.append(meta['dt'])
    return worlds, dts


#: the benchmark configurations other than the serving mix: builder of
#: ``(worlds, dts)``, the configuration's step count, and whether it is one world
CONFIGS = {
    'pyramid': (lambda api=None: (lambda r: ([r[0]], [r[1]['dt']]))(pyramid(api)), 120),
    'debris4096': (lambda api=None: (lambda r: ([r[0]], [r[1]['dt']]))(debris(api, n=4096, seed=0)), 600),
    'convex32768': (lambda api=None: (lambda r: ([r[0]], [r[1]['dt']]))(convex_pile(api, n=32768, seed=0)), 300),
    'joints512': (lambda api=None: joint_chains(512, 21, api), 480),
}
