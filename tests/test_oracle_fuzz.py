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
from fuzz_worlds import random_world, switch_worlds

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


def _step_and_compare(w, steps, name):
    o = pyoracle.OracleWorld.from_world(w)
    dt = w.fixed_dt
    n = w.body_count
    for s in range(steps):
        w.step(dt)
        o.step(dt)
        tag = '%s step %d' % (name, s)
        if w._collision is None:
            assert len(o.pairs()) == 0 and len(o.contacts()['a']) == 0, tag
            st = o.state()
            for col, key in STATE:
                assert np.array_equal(getattr(w, col)[:n], st[key]), tag + ' ' + key
            continue
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


@pytest.mark.parametrize('seed', range(4))
def test_random_world_matches_the_reference(seed):
    _step_and_compare(random_world(_ref_api(), seed), 120, 'seed %d' % seed)


def test_world_switches_match_the_reference():
    """Sleeping disabled, warm start off, default damping, no velocity
    iterations, a tilted weaker world gravity, and a world without colliders."""
    for name, w in switch_worlds(_ref_api()):
        _step_and_compare(w, 150, name)
