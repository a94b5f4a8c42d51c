"""A NaN pose written by the host between steps, through the reference and the oracle.

The reference does not guard against non-finite state: a body whose position
becomes NaN gets a NaN AABB, sorts last in the broadphase (``argsort``
places NaN after every number), overlaps nothing, and keeps integrating
(its velocity stays finite, its position NaN). The oracle must do exactly
the same, step for step, so that the device (compared with the oracle in
``test_gpu_failures.py``) is pinned to the reference's behaviour too.
Skipped when the reference is not built.
"""
import numpy as np

import pyoracle
from omi_physics_b200 import scenes
from test_oracle_fuzz import STATE, _ref_api


def _nan_world(api):
    w, meta = scenes.debris(api=api, n=48, seed=4)
    return w, meta['dt']


def test_nan_position_matches_the_reference():
    api = _ref_api()
    w, dt = _nan_world(api)
    for _ in range(30):
        w.step(dt)
    # host writes between steps, as world.position[i] = ... would
    w._position[7] = np.nan
    w._position[19, 1] = np.nan
    w._awake[19] = True
    o = pyoracle.OracleWorld.from_world(w)
    n = w.body_count
    for s in range(40):
        w.step(dt)
        o.step(dt)
        tag = 'step %d' % s
        ref_pairs = sorted(tuple(map(int, p)) for p in w._collision.broadphase.pairs(w))
        assert ref_pairs == sorted(map(tuple, o.pairs().tolist())), tag + ' pairs'
        assert all(7 not in p and 19 not in p for p in ref_pairs), tag
        st = o.state()
        for col, key in STATE:
            assert np.array_equal(getattr(w, col)[:n], st[key], equal_nan=True), tag + ' ' + key
    assert np.isnan(w._position[7]).all() and np.isfinite(w._linear_velocity[7]).all()


def test_two_bodies_nan_only_in_x_match_the_reference():
    """Two bodies whose x becomes NaN at the same height: their AABBs still
    overlap in y and z, and numpy's searchsorted puts a NaN upper bound past
    every row, so the reference pairs them (and collides them with NaN
    arithmetic). The oracle must reproduce that too."""
    api = _ref_api()
    w, dt = _nan_world(api)
    for _ in range(30):
        w.step(dt)
    w._position[11] = (np.nan, 12.0, 3.0)
    w._position[12] = (np.nan, 12.2, 3.1)
    o = pyoracle.OracleWorld.from_world(w)
    n = w.body_count
    for s in range(12):
        w.step(dt)
        o.step(dt)
        tag = 'step %d' % s
        ref_pairs = sorted(tuple(map(int, p)) for p in w._collision.broadphase.pairs(w))
        assert ref_pairs == sorted(map(tuple, o.pairs().tolist())), tag + ' pairs'
        if s == 0:
            assert (11, 12) in ref_pairs
        st = o.state()
        for col, key in STATE:
            assert np.array_equal(getattr(w, col)[:n], st[key], equal_nan=True), tag + ' ' + key
