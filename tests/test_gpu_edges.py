"""Edge cases of the step on the GPU, each against the oracle world by world.

Worlds without bodies and worlds of static bodies only, batched with the
degenerate-contact scene (coincident centres, zero-depth contacts, sleep and
wake-up) and a pyramid; a batch of empty worlds alone; and an empty world
stepped through the drop-in backend, which must behave as the reference's
step on an empty world does (nothing but the clock moves); and the wake
pass's sequential path, taken when a sleeper moving faster than the wake
threshold is among a world's contacts.
"""
import numpy as np
import pytest

import pyoracle
from omi_physics_b200 import WorldBatch, scenes
from omi_physics_b200.backend import CudaBackend

pytestmark = pytest.mark.gpu

COLS = (('_position', 'position'), ('_orientation', 'orientation'),
        ('_linear_velocity', 'linear_velocity'), ('_angular_velocity', 'angular_velocity'),
        ('_awake', 'awake'), ('_sleep_timer', 'sleep_timer'))


def _empty():
    api = scenes.default_api()
    return api.PhysicsWorld(fixed_dt=1.0 / 60.0), 1.0 / 60.0


def _statics():
    api = scenes.default_api()
    m = api.model
    w = api.PhysicsWorld(fixed_dt=1.0 / 60.0)
    slab = w.add_shape(m.Shape.box((4.0, 1.0, 4.0)))
    ball = w.add_shape(m.Shape.sphere(0.5))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=slab), position=(0.0, -0.5, 0.0))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=slab), position=(0.0, 0.2, 0.0))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ball), position=(1.0, 0.5, 1.0))
    return w, 1.0 / 60.0


def _check(b, i, w, o, tag):
    st = o.state()
    n = w.body_count
    assert np.array_equal(b.pairs(i), o.pairs()), tag + ' pairs'
    assert len(b.contacts(i)) == len(o.contacts()['a']), tag + ' contacts'
    for col, key in COLS:
        assert np.array_equal(getattr(w, col)[:n], st[key]), tag + ' ' + key


def test_empty_and_static_worlds_batched_with_degenerate_contacts():
    builders = [_empty, _statics, lambda: (lambda r: (r[0], r[1]['dt']))(scenes.degenerate()),
                _empty, lambda: (lambda r: (r[0], r[1]['dt']))(scenes.pyramid(levels=5))]
    worlds, dts = zip(*[f() for f in builders])
    oracles = [pyoracle.OracleWorld.from_world(w) for w in worlds]
    b = WorldBatch(list(worlds), dts=list(dts))
    for s in range(150):
        b.step(1)
        b.sync_to_host()
        for i, (w, o, dt) in enumerate(zip(worlds, oracles, dts)):
            o.step(dt)
            _check(b, i, w, o, 'world %d step %d' % (i, s))
    assert worlds[0].body_count == 0 and len(b.contacts(0)) == 0


def test_batch_of_empty_worlds_only():
    worlds = [_empty()[0] for _ in range(3)]
    b = WorldBatch(worlds, dts=[1.0 / 60.0] * 3)
    b.step(5)
    b.sync_to_host()
    for i in range(3):
        assert len(b.pairs(i)) == 0 and len(b.contacts(i)) == 0


def test_empty_world_through_the_drop_in_backend():
    api = scenes.default_api()
    w = api.PhysicsWorld(fixed_dt=1.0 / 60.0, backend=CudaBackend())
    for _ in range(4):
        w.step(1.0 / 60.0)
    assert w.body_count == 0 and len(w.contacts) == 0
    assert w.time == pytest.approx(4.0 / 60.0)


def test_wake_cascade_from_a_moving_sleeper():
    """A sleeping body that carries velocity (written by the host while it
    sleeps) meets the kinematic pusher: the wake pass finds a sleeper faster
    than the wake threshold among the contacts and resolves that world in the
    reference's sequential contact order (solver.py:321-337). The velocity is
    set on the resting row of the degenerate scene just before the pusher's
    first contact; every following step equals the oracle bit for bit."""
    row = [15, 16, 17, 18]
    probe, meta = scenes.degenerate()
    dt = meta['dt']
    po = pyoracle.OracleWorld.from_world(probe)
    first = None
    for s in range(200):
        po.step(dt)
        c = po.contacts()
        if any((int(a), int(b)) == (18, 19) for a, b in zip(c['a'], c['b'])):
            first = s
            break
    assert first is not None
    w, _ = scenes.degenerate()
    o = pyoracle.OracleWorld.from_world(w)
    b = WorldBatch([w], dts=[dt])
    b.step(first)
    for _ in range(first):
        o.step(dt)
    b.sync_to_host()
    _check(b, 0, w, o, 'before the pusher')
    assert not w._awake[row].any()
    for i in row:
        w._linear_velocity[i] = (-0.3, 0.0, 0.0)
        o.set_linear_velocity(i, (-0.3, 0.0, 0.0))
    b.upload_state(0)
    for s in range(40):
        b.step(1)
        b.sync_to_host()
        o.step(dt)
        _check(b, 0, w, o, 'cascade step %d' % s)
        if s == 0:
            assert w._awake[row].all()          # the pusher woke the whole moving row
