"""Host paths on the GPU: buffer regrowth on overflow (synchronous and
asynchronous steps), the warm-start cache round trip, snapshot / restore of a
world (state + warm-start cache + sensor overlaps) in a batch and in a
serving slot, sensor worlds batched with plain ones, and serving slots
refusing sensor worlds."""
import numpy as np
import pytest

import pyoracle
from omi_physics_b200 import WorldBatch, scenes
from omi_physics_b200._lib import OmiError
from omi_physics_b200.serving import Server, size_classes

pytestmark = pytest.mark.gpu

COLS = ('_position', '_orientation', '_linear_velocity', '_angular_velocity', '_awake', '_sleep_timer')


def _dense(seed=7):
    # 300 bodies packed into a few cubic metres: far more candidate pairs than
    # the arena's first pair buffer (4096) and contacts than its contact buffer
    return scenes.debris(n=300, seed=seed, extent=1.5, height=2.0, ground=10.0)


def _equal_state(w, o, tag):
    st = o.state()
    n = w.body_count
    for col, key in zip(COLS, ('position', 'orientation', 'linear_velocity', 'angular_velocity',
                               'awake', 'sleep_timer')):
        assert np.array_equal(getattr(w, col)[:n], st[key]), tag + col


def test_overflow_regrows_and_matches_oracle():
    w, meta = _dense()
    dt = meta['dt']
    o = pyoracle.OracleWorld.from_world(w)
    b = WorldBatch([w], dts=[dt])
    for s in range(3):
        b.step(1)
        o.step(dt)
        b.sync_to_host()
        if s == 0:                           # the packed start overflows the first buffers
            p, c = b.counts()
            assert p[0] > 4096 and c[0] > 0
        assert np.array_equal(b.pairs(0), o.pairs()), s
        _equal_state(w, o, 'step %d ' % s)


def test_async_overflow_reported_then_recovered():
    w, meta = _dense(seed=8)
    dt = meta['dt']
    n = w.body_count
    before = {col: np.array(getattr(w, col)[:n], copy=True) for col in COLS}
    o = pyoracle.OracleWorld.from_world(w)
    b = WorldBatch([w], dts=[dt])
    b.step_async(1)
    with pytest.raises(OmiError):
        b.sync()
    b.sync_to_host()
    for col in COLS:                         # the overflowing step changed nothing
        assert np.array_equal(getattr(w, col)[:n], before[col]), col
    b.step(1)                                # grows the buffers and runs the step
    o.step(dt)
    b.sync_to_host()
    _equal_state(w, o, 'after recovery ')


def test_cache_round_trip():
    w, meta = scenes.pyramid()
    b = WorldBatch([w], dts=[meta['dt']])
    b.step(12)
    c = b.cache(0)
    assert len(c['a']) > 0
    b.set_cache(0, c['a'], c['b'], c['point'], c['impulse'])
    c2 = b.cache(0)
    for k in ('a', 'b', 'point', 'impulse'):
        assert np.array_equal(c[k], c2[k]), k


def test_snapshot_restore_continues_identically():
    w1, meta = scenes.debris(n=400, seed=21, extent=5.0, height=6.0, ground=20.0)
    dt = meta['dt']
    b1 = WorldBatch([w1], dts=[dt])
    b1.step(60)
    snap = b1.snapshot(0)
    b1.step(30)
    b1.sync_to_host()
    w2, _ = scenes.debris(n=400, seed=21, extent=5.0, height=6.0, ground=20.0)
    b2 = WorldBatch([w2], dts=[dt])
    b2.restore(0, snap)
    b2.step(30)
    b2.sync_to_host()
    n = w1.body_count
    for col in COLS:
        assert np.array_equal(getattr(w1, col)[:n], getattr(w2, col)[:n]), col


def test_serving_snapshot_restore():
    srv = Server(size_classes(256, per_class=2, min_bodies=64))
    w, meta = scenes.debris(n=150, seed=31, extent=3.0, height=4.0, ground=12.0)
    req = srv.submit(w, steps=40, dt=meta['dt'], arrival=0)
    for t in range(10):
        srv.tick(float(t))
    snap = srv.snapshot(req)
    for t in range(10, 20):
        srv.tick(float(t))
    later = srv.snapshot(req)
    srv.restore(req, snap)
    for t in range(10, 20):
        srv.tick(float(t))
    again = srv.snapshot(req)
    for k in ('pos', 'q', 'v', 'w', 'awake', 'timer'):
        assert np.array_equal(later[k], again[k]), k
    srv.close()


def test_world_groups_equal_one_batch():
    from omi_physics_b200.groups import WorldGroups
    reqs = scenes.serving_requests(16, seed=9, n_min=16, n_max=256)
    one = [scenes.serving_world(r)[0] for r in reqs]
    many = [scenes.serving_world(r)[0] for r in reqs]
    b = WorldBatch(one)
    g = WorldGroups(many, groups=3)
    b.step(30)
    g.step(20)
    g.step_async(10)
    g.sync()
    b.sync_to_host()
    g.sync_to_host()
    for w1, w2 in zip(one, many):
        n = w1.body_count
        for col in COLS:
            assert np.array_equal(getattr(w1, col)[:n], getattr(w2, col)[:n]), col
    # the host round trip of the groups equals plain steps too
    bufs = g.host_buffers()
    from omi_physics_b200._lib import D, U8, ptr
    for bt, h in zip(g.batches, bufs):
        nb = bt.packed.n_bodies
        bt.ctx.call('download_state', 0, nb, ptr(h['pos'], D), ptr(h['q'], D), ptr(h['v'], D), ptr(h['w'], D),
                    ptr(h['awake'], U8), ptr(h['timer'], D), None, None)
    g.step_from_host(bufs, 2)
    b.step(2)
    b.sync_to_host()
    g.sync_to_host()
    for w1, w2 in zip(one, many):
        n = w1.body_count
        assert np.array_equal(w1._position[:n], w2._position[:n])
    g.close()


def _oracle_events(o, prev):
    new = o.overlaps()
    ev = ([('enter',) + p for p in sorted(new - prev)] + [('stay',) + p for p in sorted(new & prev)] +
          [('exit',) + p for p in sorted(prev - new)])
    return new, ev


def test_sensor_worlds_in_a_batch_match_the_oracle():
    """Three sensor / gravity-volume worlds and a plain one stepped together:
    every world's per-step trigger events and final state equal the oracle's
    for that world alone."""
    def build():
        return [scenes.zones(n=80 + 20 * k, seed=k) for k in range(3)] + \
               [scenes.debris(n=100, seed=5, extent=4.0, height=5.0, ground=16.0)]
    worlds = [w for w, _ in build()]
    b = WorldBatch(worlds, dts=[1 / 120.0] * 4)
    assert b.has_sensors
    refs = [pyoracle.OracleWorld.from_world(w) for w, _ in build()]
    prev = [set() for _ in refs]
    want = [[] for _ in refs]
    for _ in range(80):
        b.step(1)
        for k, o in enumerate(refs):
            o.step(1 / 120.0)
            prev[k], ev = _oracle_events(o, prev[k])
            want[k].extend(ev)
    b.sync_to_host()
    for k, (w, o) in enumerate(zip(worlds, refs)):
        assert b.take_events(k) == want[k], k
        _equal_state(w, o, 'world %d ' % k)
    assert len(want[0]) > 50 and not want[3]


def test_sensor_snapshot_restore_continues_identically():
    w1, meta = scenes.zones(n=120, seed=8)
    b1 = WorldBatch([w1], dts=[meta['dt']])
    b1.step(40)
    snap = b1.snapshot(0)
    b1.take_events(0)
    b1.step(30)
    ev1 = b1.take_events(0)
    b1.sync_to_host()
    w2, _ = scenes.zones(n=120, seed=8)
    b2 = WorldBatch([w2], dts=[meta['dt']])
    b2.restore(0, snap)
    b2.step(30)
    assert b2.take_events(0) == ev1 and ev1
    b2.sync_to_host()
    n = w1.body_count
    for col in COLS:
        assert np.array_equal(getattr(w1, col)[:n], getattr(w2, col)[:n]), col


def test_serving_slots_refuse_sensor_and_mesh_worlds():
    from omi_physics_b200._lib import UnsupportedFeature
    srv = Server(size_classes(256, per_class=1, min_bodies=64))
    w, meta = scenes.zones(n=60, seed=2)
    with pytest.raises(UnsupportedFeature):
        srv.submit(w, steps=5, dt=meta['dt'], arrival=0)
    w, meta = scenes.terrain(n=20, seed=2, cells=8, extent=3.0)
    with pytest.raises(UnsupportedFeature):
        srv.submit(w, steps=5, dt=meta['dt'], arrival=0)
    srv.close()
