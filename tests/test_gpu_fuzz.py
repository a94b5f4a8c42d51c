"""The seeded random worlds of the fuzz tests on the GPU: eight of them in one
batch (uneven sizes, sensors, gravity volumes, every shape kind and motion
type), 120 steps, each world's pairs, contacts, impulses, state, sleep flags
and sensor overlaps equal to the oracle's for that world alone, bit for bit,
at every step. The oracle itself matches the reference on the same worlds
(``tests/test_oracle_fuzz.py``)."""
import numpy as np
import pytest

import pyoracle
from fuzz_worlds import random_world, switch_worlds
from omi_physics_b200 import WorldBatch, scenes

pytestmark = pytest.mark.gpu

STATE = (('_position', 'position'), ('_orientation', 'orientation'),
         ('_linear_velocity', 'linear_velocity'), ('_angular_velocity', 'angular_velocity'),
         ('_awake', 'awake'), ('_sleep_timer', 'sleep_timer'))


def _batched_against_oracles(worlds, steps):
    oracles = [pyoracle.OracleWorld.from_world(w) for w in worlds]
    b = WorldBatch(worlds, dts=[w.fixed_dt for w in worlds])
    for s in range(steps):
        b.step(1)
        b.sync_to_host()
        for i, (w, o) in enumerate(zip(worlds, oracles)):
            o.step(w.fixed_dt)
            tag = 'world %d step %d' % (i, s)
            assert np.array_equal(b.pairs(i), o.pairs()), tag + ' pairs'
            c, oc = b.contact_arrays(i), o.contacts()
            for key in ('a', 'b', 'point', 'normal', 'depth', 'impulse'):
                assert np.array_equal(c[key], oc[key]), tag + ' contact ' + key
            st = o.state()
            n = w.body_count
            for col, key in STATE:
                assert np.array_equal(getattr(w, col)[:n], st[key]), tag + ' ' + key
            assert b.trigger_overlaps(i) == o.overlaps(), tag + ' overlaps'


def test_random_worlds_batched_match_the_oracle():
    api = scenes.default_api()
    _batched_against_oracles([random_world(api, seed) for seed in range(8)], 120)


def test_world_switches_batched_match_the_oracle():
    """Sleeping disabled, warm start off (contacts report zero impulses, as the
    reference leaves them), default damping, no velocity iterations, a tilted
    weaker world gravity and a world without colliders, in one batch."""
    _batched_against_oracles([w for _, w in switch_worlds(scenes.default_api())], 150)
