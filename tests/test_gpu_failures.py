"""Failure paths of the device step, made to happen on purpose and without a fault.

* A contact-sweep wait that runs out: ``omi_set_limits`` lowers the wait
  bound and stalls one run (its entries ask for more arrivals than they can
  get), so the sweep's bounded waits give up. The kernel returns, the rest of
  the step does nothing, and the step reports OMI_E_TIMEOUT
  (:class:`SweepTimeout`). The context stays usable: with the limits back at
  their defaults and the world restored from a snapshot, the next steps match
  the oracle bit for bit.
* An EPA polytope that outgrows its bound: with the face bound lowered to 4,
  every convex pair that reaches EPA overflows; the step completes, drops
  those contacts and reports OMI_E_LIMIT (:class:`EpaLimit`), the only way a
  caller learns that the step differs from the reference's unbounded EPA.
* A NaN pose written by the host between steps, and two bodies whose x alone
  becomes NaN (the reference then pairs them, as numpy's searchsorted puts a
  NaN bound past every row): the device follows the oracle, which follows
  the reference (``test_oracle_nan.py``), NaNs included.
* A malformed scene (a shape index out of range) is refused by ``omi_load``
  before the previous arena is released: the worlds loaded before keep
  stepping, bit-exact with the oracle.
"""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from omi_physics_b200 import WorldBatch, scenes
from omi_physics_b200._lib import EpaLimit, OmiError, SweepTimeout, OMI_E_ARG
from omi_physics_b200.arena import pack_worlds

pytestmark = pytest.mark.gpu

COLS = (('_position', 'position'), ('_orientation', 'orientation'),
        ('_linear_velocity', 'linear_velocity'), ('_angular_velocity', 'angular_velocity'),
        ('_awake', 'awake'), ('_sleep_timer', 'sleep_timer'))


def _check(b, w, o, tag, nan=False):
    st = o.state()
    n = w.body_count
    assert np.array_equal(b.pairs(0), o.pairs()), tag + ' pairs'
    c, oc = b.contact_arrays(0), o.contacts()
    assert np.array_equal(c['a'], oc['a']) and np.array_equal(c['b'], oc['b']), tag + ' contacts'
    for k in ('point', 'normal', 'depth', 'impulse'):
        assert np.array_equal(c[k], oc[k], equal_nan=nan), tag + ' contact ' + k
    for col, key in COLS:
        assert np.array_equal(getattr(w, col)[:n], st[key], equal_nan=nan), tag + ' ' + key


def _oracle_at(b, w, i=0):
    """An oracle world at the batch's current state, warm-start cache included."""
    b.sync_to_host()
    o = pyoracle.OracleWorld.from_world(w)
    c = b.cache(i)
    o.set_cache(c['a'], c['b'], c['point'], c['impulse'])
    return o


def test_sweep_wait_that_runs_out_fails_the_step_and_the_context_recovers():
    w, meta = scenes.pyramid()
    dt = meta['dt']
    b = WorldBatch([w], dts=[dt])
    b.step(6)                                    # the pyramid is in contact, every box awake
    assert b.counts()[1][0] > 100
    snap = b.snapshot(0)
    b.ctx.set_limits(spin_limit=20000, stall_run=0)
    with pytest.raises(SweepTimeout) as e:
        b.step(1)
    assert 'timed out' in str(e.value)
    # the context is usable: defaults back, state restored, stepping matches the oracle
    b.ctx.set_limits()
    b.restore(0, snap)
    o = _oracle_at(b, w)
    for s in range(12):
        b.step(1)
        o.step(dt)
        b.sync_to_host()
        _check(b, w, o, 'after timeout, step %d' % s)


def test_epa_face_bound_reports_the_dropped_contacts():
    w, meta = scenes.convex_pile(n=300, seed=2, arena=14.0, height=6.0)
    dt = meta['dt']
    b = WorldBatch([w], dts=[dt])
    b.step(40)                                   # hulls resting on each other and the floor
    snap = b.snapshot(0)
    o = _oracle_at(b, w)
    o.step(dt)
    full = len(o.contacts()['a'])
    b.ctx.set_limits(epa_faces=4)
    with pytest.raises(EpaLimit) as e:
        b.step(1)
    assert 'EPA' in str(e.value)
    assert len(b.contact_arrays(0)['a']) < full     # the step completed without those contacts
    b.ctx.set_limits()
    b.restore(0, snap)
    o = _oracle_at(b, w)
    for s in range(5):
        b.step(1)
        o.step(dt)
        b.sync_to_host()
        _check(b, w, o, 'after the EPA limit, step %d' % s)


def test_nan_poses_follow_the_oracle():
    w, meta = scenes.debris(n=48, seed=4)
    dt = meta['dt']
    b = WorldBatch([w], dts=[dt])
    b.step(30)
    b.sync_to_host()
    w._position[7] = np.nan
    w._position[19, 1] = np.nan
    w._awake[19] = True
    w._position[11] = (np.nan, 12.0, 3.0)        # x alone NaN: the reference pairs 11 and 12
    w._position[12] = (np.nan, 12.2, 3.1)
    b.upload_state(0)
    o = _oracle_at(b, w)
    for s in range(30):
        b.step(1)
        o.step(dt)
        b.sync_to_host()
        _check(b, w, o, 'NaN step %d' % s, nan=True)
        if s == 0:
            assert (11, 12) in set(map(tuple, b.pairs(0).tolist()))


def test_malformed_scene_is_refused_and_the_loaded_worlds_keep_stepping():
    w, meta = scenes.debris(n=64, seed=9)
    dt = meta['dt']
    b = WorldBatch([w], dts=[dt])
    b.step(20)
    o = _oracle_at(b, w)
    bad_world, _ = scenes.debris(n=16, seed=1)
    P = pack_worlds([bad_world], [dt])
    P.arrays['shape'][3] = P.scene.n_shapes + 4
    with pytest.raises(OmiError) as e:
        b.ctx.call('load', C.byref(P.scene))
    assert e.value.code == OMI_E_ARG and 'shape index' in str(e.value)
    for s in range(10):
        b.step(1)
        o.step(dt)
        b.sync_to_host()
        _check(b, w, o, 'after a refused load, step %d' % s)
