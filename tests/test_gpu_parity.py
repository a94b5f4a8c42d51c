"""GPU parity through the C ABI.

(1) Golden checkpoints: the reference's own one-step inputs (state, joint
state, warm-start cache) replayed on the B200 must give the reference's
pairs, contacts, impulses, poses, sleep flags and sensor overlaps / events — bit for bit on the
box/sphere/convex/capsule scenes (the kernels keep the reference's arithmetic order
and are built with --fmad=false), within 1e-12 relative on the joint scene
(the reference solves point joints with LAPACK).
(2) Trajectories against the oracle, every step, at sizes the oracle runs in
seconds: pair lists, contacts, impulses, sleep islands and state bit-exact.
"""
import numpy as np
import pytest

import pyoracle
from golden_util import SCENES, checkpoints, events_from_overlaps, load, pair_set
from omi_physics_b200 import WorldBatch, scenes
from util import assert_close, world_at_checkpoint

pytestmark = pytest.mark.gpu

EXACT = {'pyramid', 'debris', 'convex', 'spheres', 'capsules', 'zones', 'terrain', 'ridge', 'conveyor',
         'degenerate', 'rods'}


@pytest.mark.parametrize('scene', SCENES)
def test_golden_checkpoints_on_gpu(scene):
    rel = 0 if scene in EXACT else 1e-12
    for step in checkpoints(load(scene)):
        w, dt, ins, outs = world_at_checkpoint(scene, step)
        b = WorldBatch([w], dts=[dt])
        b.set_cache(0, ins['cache_a'], ins['cache_b'], ins['cache_point'], ins['cache_impulse'])
        b.step(1)
        b.sync_to_host()
        tag = '%s@%d' % (scene, step)
        assert np.array_equal(b.pairs(0), outs['pairs']), tag + ' pairs'
        c = b.contact_arrays(0)
        assert np.array_equal(np.stack([c['a'], c['b']], 1).reshape(-1, 2), outs['c_ab']), tag
        assert_close(c['point'], outs['c_point'], rel, tag + ' point')
        assert_close(c['normal'], outs['c_normal'], rel, tag + ' normal')
        assert_close(c['depth'], outs['c_depth'], rel, tag + ' depth')
        assert_close(c['impulse'], outs['c_impulse'], rel, tag + ' impulse')
        n = w.body_count
        for col, key in (('position', 'position'), ('orientation', 'orientation'),
                         ('linear_velocity', 'linear_velocity'),
                         ('angular_velocity', 'angular_velocity'), ('sleep_timer', 'sleep_timer'),
                         ('aabb_min', 'aabb_min'), ('aabb_max', 'aabb_max')):
            assert_close(getattr(w, col), outs[key], rel, tag + ' ' + col)
        assert np.array_equal(w.awake, outs['awake'].astype(bool)), tag + ' awake'
        if 'overlaps' in outs:
            new = b.trigger_overlaps(0)
            assert new == pair_set(outs['overlaps']), tag + ' trigger overlaps'
            ev = events_from_overlaps(pair_set(ins['overlaps_prev']), new)
            assert np.array_equal(ev, outs['events']), tag + ' trigger events'


def _compare_step(b, w, o, tag):
    st = o.state()
    assert np.array_equal(b.pairs(0), o.pairs()), tag + ' pairs'
    c, oc = b.contact_arrays(0), o.contacts()
    assert np.array_equal(c['a'], oc['a']) and np.array_equal(c['b'], oc['b']), tag + ' ab'
    for key in ('point', 'normal', 'depth', 'impulse'):
        assert np.array_equal(c[key], oc[key]), tag + ' ' + key
    for col in ('position', 'orientation', 'linear_velocity', 'angular_velocity', 'sleep_timer',
                'aabb_min', 'aabb_max'):
        assert np.array_equal(getattr(w, col), st[col]), tag + ' ' + col
    assert np.array_equal(w.awake, st['awake']), tag + ' awake'
    assert o.islands() == _island_sets(b.islands(0)), tag + ' islands'
    if b.has_sensors:
        assert b.trigger_overlaps(0) == o.overlaps(), tag + ' trigger overlaps'


def _island_sets(labels):
    groups = {}
    for i, l in enumerate(labels):
        if l >= 0:
            groups.setdefault(int(l), set()).add(i)
    return {frozenset(g) for g in groups.values()}


@pytest.mark.parametrize('name,builder,steps', [
    ('pyramid', lambda: scenes.pyramid(), 120),
    ('debris512', lambda: scenes.debris(n=512, seed=1, extent=8.0, height=12.0, ground=30.0), 150),
    ('convex160', lambda: scenes.convex_pile(n=160, seed=2, arena=10.0, height=8.0), 150),
    ('feature_mix', lambda: scenes.feature_mix(), 120),
    ('capsules256', lambda: scenes.capsule_pile(n=256, seed=3, arena=12.0, height=8.0), 150),
    ('zones300', lambda: scenes.zones(n=300, seed=4, extent=6.0, height=10.0), 150),
    ('terrain150', lambda: scenes.terrain(n=150, seed=2, cells=30, extent=8.0), 150),
    ('conveyor120', lambda: scenes.conveyor(n=120, seed=3, cells=20, extent=6.0), 150),
    ('degenerate', lambda: scenes.degenerate(), 300),
    ('rods', lambda: scenes.rods(), 240),
])
def test_trajectory_matches_oracle_every_step(name, builder, steps):
    w, meta = builder()
    dt = meta['dt']
    o = pyoracle.OracleWorld.from_world(w)
    b = WorldBatch([w], dts=[dt])
    for s in range(steps):
        b.step(1)
        b.sync_to_host()
        o.step(dt)
        _compare_step(b, w, o, '%s step %d' % (name, s))


def test_joint_chain_trajectory_within_tolerance():
    w, meta = scenes.joint_chain(links=24, loose=32, seed=4)
    dt = meta['dt']
    o = pyoracle.OracleWorld.from_world(w)
    b = WorldBatch([w], dts=[dt])
    for s in range(60):
        b.step(1)
        o.step(dt)
    b.sync_to_host()
    st = o.state()
    assert float(np.max(np.abs(w.position - st['position']))) < 1e-6
    assert float(np.max(np.abs(w.orientation - st['orientation']))) < 1e-6


def test_serving_mix_batch_matches_oracle_per_world():
    """64 worlds of the serving mix (uneven sizes) stepped together for 120 steps:
    every world's pairs, poses, velocities and sleep flags equal the oracle's
    for that world alone, bit for bit."""
    reqs = scenes.serving_requests(64, seed=0)
    worlds, dts = [], []
    for r in reqs:
        w, meta = scenes.serving_world(r)
        worlds.append(w)
        dts.append(meta['dt'])
    b = WorldBatch(worlds, dts=dts)
    b.step(120)
    b.sync_to_host()
    for i, r in enumerate(reqs):
        w0, meta = scenes.serving_world(r)
        o = pyoracle.OracleWorld.from_world(w0)
        for _ in range(120):
            o.step(meta['dt'])
        st = o.state()
        w = worlds[i]
        n = w.body_count
        assert np.array_equal(b.pairs(i), o.pairs()), (i, 'pairs')
        assert np.array_equal(w._position[:n], st['position']), (i, 'position')
        assert np.array_equal(w._orientation[:n], st['orientation']), (i, 'orientation')
        assert np.array_equal(w._linear_velocity[:n], st['linear_velocity']), (i, 'v')
        assert np.array_equal(w._angular_velocity[:n], st['angular_velocity']), (i, 'w')
        assert np.array_equal(w._awake[:n], st['awake']), (i, 'awake')
