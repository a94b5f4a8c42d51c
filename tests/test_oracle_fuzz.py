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
from fuzz_worlds import joint_world, random_world, switch_worlds

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
    from omi_physics import gravity, joints, model
    return SimpleNamespace(PhysicsWorld=ref.PhysicsWorld, model=model, gravity=gravity, joints=joints)


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


@pytest.mark.parametrize('seed', range(4))
def test_random_joint_world_matches_the_reference(seed):
    """Point joints (the reference solves each with LAPACK, the oracle with a
    partial-pivot LU: ~1e-15 apart per solve) between bodies and to the world,
    distance joints and motors: 60 steps, pair lists exact, poses and velocities
    within 1e-9, the lazily fixed joint state within 1e-9."""
    w = joint_world(_ref_api(), seed)
    o = pyoracle.OracleWorld.from_world(w)
    n = w.body_count
    for s in range(60):
        w.step(w.fixed_dt)
        o.step(w.fixed_dt)
        tag = 'seed %d step %d' % (seed, s)
        ref_pairs = sorted(tuple(map(int, p)) for p in w._collision.broadphase.pairs(w))
        assert ref_pairs == sorted(map(tuple, o.pairs().tolist())), tag + ' pairs'
        st = o.state()
        for col, key in STATE[:4]:
            assert np.allclose(getattr(w, col)[:n], st[key], rtol=0, atol=1e-9), tag + ' ' + key
        assert np.array_equal(w._awake[:n], st['awake']), tag + ' awake'
    js = o.joint_state()
    for j, c in enumerate(w.joint_constraints):
        if hasattr(c, 'local_a'):                       # point joint: the world side stays None
            for attr in ('local_a', 'local_b'):
                if getattr(c, attr) is not None:
                    assert np.allclose(getattr(c, attr), js[attr][j], rtol=0, atol=1e-9), (j, attr)
        elif hasattr(c, 'length'):
            assert abs(c.length - js['length'][j]) <= 1e-9, j
        elif hasattr(c, 'accum'):
            assert abs(c.accum - js['accum'][j]) <= 1e-9, j
