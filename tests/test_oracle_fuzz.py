"""Seeded random worlds through the reference and the oracle, every step.

Each world mixes what the step's routes and tables branch on: boxes,
spheres, capsules, cylinders and hulls; static, kinematic (moving, turning)
and dynamic bodies, some without a collider, and a resting stack that falls
asleep; materials with every friction and restitution combine mode and a
pair-friction override; collision filters; damping, quadratic drag and
gravity factors; sensors on static, kinematic and dynamic bodies; and
gravity volumes of every kind and behaviour. The reference (built from its
sources into ``oracle/_ref``) and the oracle step the same world; pair lists,
contacts (pairs, points, normals, depths, impulses), poses, velocities, sleep
state and sensor overlaps must agree bit for bit at every step. Joints are
left out here: the reference solves point joints with LAPACK, which the
oracle matches to ~1e-12, not bit for bit. Skipped when the reference is not
built.
"""
import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

import pyoracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, 'oracle', '_ref')
STATE = (('_position', 'position'), ('_orientation', 'orientation'),
         ('_linear_velocity', 'linear_velocity'), ('_angular_velocity', 'angular_velocity'),
         ('_awake', 'awake'), ('_sleep_timer', 'sleep_timer'))


def _ref_api():
    if not os.path.isdir(os.path.join(REF, 'omi_physics')):
        pytest.skip('the reference is not built (oracle/build_ref.sh)')
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import omi_physics as ref
    from omi_physics import gravity, model
    return SimpleNamespace(PhysicsWorld=ref.PhysicsWorld, model=model, gravity=gravity)


def _quat(rng):
    q = rng.normal(size=4)
    return tuple(float(x) for x in q / np.linalg.norm(q))


def random_world(api, seed, n=40):
    m, G = api.model, api.gravity
    rng = np.random.default_rng(seed)
    w = api.PhysicsWorld(fixed_dt=1.0 / 120.0, default_linear_damping=float(rng.choice([0.0, 0.02])))
    modes = (m.AVERAGE, m.MINIMUM, m.MAXIMUM, m.MULTIPLY)
    mats = [w.add_material(m.Material(staticFriction=float(rng.uniform(0.1, 1.0)),
                                      dynamicFriction=float(rng.uniform(0.05, 0.9)),
                                      restitution=float(rng.choice([0.0, 0.2, 0.7])),
                                      frictionCombine=modes[k % 4], restitutionCombine=modes[(k + 1) % 4]))
            for k in range(5)]
    w.set_pair_friction(mats[0], mats[1], 0.8, 0.7)
    filters = [-1,
               w.add_filter(m.CollisionFilter(collisionSystems=('a',), notCollideWithSystems=('b',))),
               w.add_filter(m.CollisionFilter(collisionSystems=('b',))),
               w.add_filter(m.CollisionFilter(collisionSystems=('c',), collideWithSystems=('c', 'a')))]
    ground = w.add_shape(m.Shape.box((14.0, 1.0, 14.0)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ground, physicsMaterial=mats[0]),
               position=(0.0, -0.5, 0.0))

    def shape():
        k = rng.integers(0, 5)
        if k == 0:
            return w.add_shape(m.Shape.box(tuple(float(x) for x in rng.uniform(0.3, 1.4, 3))))
        if k == 1:
            return w.add_shape(m.Shape.sphere(float(rng.uniform(0.2, 0.7))))
        if k == 2:
            return w.add_shape(m.Shape.capsule(float(rng.uniform(0.3, 1.2)), float(rng.uniform(0.15, 0.4))))
        if k == 3:
            return w.add_shape(m.Shape.cylinder(float(rng.uniform(0.4, 1.2)), float(rng.uniform(0.2, 0.5))))
        pts = rng.normal(size=(int(rng.integers(8, 20)), 3))
        pts *= rng.uniform(0.3, 0.8, 3) / np.linalg.norm(pts, axis=1, keepdims=True)
        return w.add_shape(m.Shape.convex(pts))

    for i in range(n):
        u = rng.random()
        kind = m.STATIC if u < 0.08 else (m.KINEMATIC if u < 0.16 else m.DYNAMIC)
        pos = tuple(float(x) for x in rng.uniform((-2.5, 0.3, -2.5), (2.5, 3.0, 2.5)))
        motion = m.Motion(type=kind, mass=float(rng.uniform(0.5, 4.0)),
                          linearVelocity=tuple(float(x) for x in rng.normal(0.0, 0.6, 3)) if kind != m.STATIC
                          else (0.0, 0.0, 0.0),
                          angularVelocity=tuple(float(x) for x in rng.normal(0.0, 0.4, 3)) if kind != m.STATIC
                          else (0.0, 0.0, 0.0),
                          linearDamping=float(rng.choice([0.0, 0.1])), angularDamping=float(rng.choice([0.0, 0.2])),
                          quadraticDrag=float(rng.choice([0.0, 0.03])), gravityFactor=float(rng.choice([1.0, 0.5, 1.5])))
        collider = None if rng.random() < 0.05 else m.Collider(shape=shape(), physicsMaterial=mats[i % 5],
                                                              collisionFilter=filters[i % 4])
        trigger = m.Trigger(shape=shape()) if rng.random() < 0.12 else None
        if collider is None and trigger is None and kind == m.STATIC:
            continue
        w.add_body(motion, collider, trigger=trigger, position=pos, orientation=_quat(rng))
    unit = w.add_shape(m.Shape.box((1.0, 1.0, 1.0)))
    for k in range(4):                  # a resting stack that falls asleep unless something hits it
        w.add_body(m.Motion(type=m.DYNAMIC), m.Collider(shape=unit, physicsMaterial=mats[0]),
                   position=(5.5, 0.5 + k, 5.5))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(type='point', gravity=5.0, center=(2.0, 2.0, 0.0), priority=1),
                                         G.SphereRegion((2.0, 2.0, 0.0), 2.5)))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(gravity=3.0, direction=(0.3, 1.0, 0.0), priority=2,
                                                   replace=True), G.BoxRegion((-2.5, 2.0, 2.5), (1.5, 2.0, 1.5))))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(priority=3, stop=True), G.BoxRegion((2.5, 1.5, -2.5), (1.0, 1.5, 1.0))))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(gravity=0.4, direction=(0.0, 0.0, 1.0))))
    w._collision.solver.velocity_iterations = int(rng.integers(4, 11))
    return w


@pytest.mark.parametrize('seed', range(4))
def test_random_world_matches_the_reference(seed):
    api = _ref_api()
    w = random_world(api, seed)
    o = pyoracle.OracleWorld.from_world(w)
    dt = w.fixed_dt
    n = w.body_count
    for s in range(120):
        w.step(dt)
        o.step(dt)
        tag = 'seed %d step %d' % (seed, s)
        ref_pairs = sorted(tuple(map(int, p)) for p in w._collision.broadphase.pairs(w))
        assert ref_pairs == sorted(map(tuple, o.pairs().tolist())), tag + ' pairs'
        c = o.contacts()
        rc = w.contacts
        assert len(rc) == len(c['a']), tag + ' contact count'
        for k, x in enumerate(rc):
            assert (int(x.a), int(x.b)) == (int(c['a'][k]), int(c['b'][k])), tag + ' contact pair'
            assert np.array_equal(x.point, c['point'][k]) and np.array_equal(x.normal, c['normal'][k]), tag
            assert x.depth == c['depth'][k], tag + ' depth'
            imp = np.array([x.normal_impulse, *x.tangent_impulse])
            assert np.array_equal(imp, c['impulse'][k]), tag + ' impulse'
        st = o.state()
        for col, key in STATE:
            assert np.array_equal(getattr(w, col)[:n], st[key]), tag + ' ' + key
        assert set(w._collision.triggers.overlaps) == o.overlaps(), tag + ' overlaps'
