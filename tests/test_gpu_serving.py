"""Serving on the GPU: requests admitted into slots while others step, each
world's result the same as stepping it alone.

Worlds are independent and every kernel works world by world (own sort, own
pairs, own levels, own warm-start cache), so residency with other worlds
changes nothing: final state alone vs in the mix is compared bit for bit
(the 1e-9 one-step / 1e-6 m trajectory tolerances are therefore met with
zero difference), and one world is checked against the oracle.
"""
import numpy as np
import pytest

import pyoracle
from omi_physics_b200 import WorldBatch, scenes
from omi_physics_b200.serving import Server, size_classes

pytestmark = pytest.mark.gpu

STATE = ('_position', '_orientation', '_linear_velocity', '_angular_velocity', '_awake', '_sleep_timer')


def _requests():
    reqs = scenes.serving_requests(10, seed=3, n_min=16, n_max=96)
    return [(r, 18 + (7 * i) % 25, 2 * i) for i, r in enumerate(reqs)]


def test_serving_results_match_alone_and_oracle():
    plan = _requests()
    srv = Server(size_classes(96, per_class=3, min_bodies=32))     # 9 slots for 10 requests
    subs = []
    for r, steps, arrival in plan:
        w, meta = scenes.serving_world(r)
        subs.append(srv.submit(w, steps, dt=meta['dt'], arrival=arrival))
    stats = srv.run(clock='ticks')
    assert stats.completed == len(plan)
    assert stats.peak_active >= 3                  # overlap: several worlds resident at once
    slots = [q.slot for q in subs]
    assert len(set(slots)) < len(slots)            # 10 requests through 9 slots: one was reused
    for (r, steps, _), q in zip(plan, subs):
        w, meta = scenes.serving_world(r)
        b = WorldBatch([w], dts=[meta['dt']])
        b.step(steps)
        b.sync_to_host()
        for col in STATE:
            assert np.array_equal(getattr(q.world, col)[:w.body_count], getattr(w, col)[:w.body_count]), \
                (q.rid, col)
    # one of them against the oracle
    r, steps, _ = plan[4]
    w, meta = scenes.serving_world(r)
    o = pyoracle.OracleWorld.from_world(w)
    for _ in range(steps):
        o.step(meta['dt'])
    st = o.state()
    assert np.array_equal(subs[4].world._position[:w.body_count], st['position'])
    assert np.array_equal(subs[4].world._orientation[:w.body_count], st['orientation'])
    assert np.array_equal(subs[4].world._awake[:w.body_count], st['awake'])
    srv.close()


def test_serving_budget_refuses_oversized_reservation():
    from omi_physics_b200._lib import OutOfBudget
    with pytest.raises(OutOfBudget):
        Server(size_classes(2048, per_class=64), budget_bytes=64 << 20)


def test_serving_an_omi_document():
    """An OMI glTF document (no sensors or volumes) served through a slot ends
    where the oracle, stepping the world built from the same document, ends."""
    import json
    from golden_util import GOLDEN
    from omi_physics_b200 import gltf
    doc = json.load(open(GOLDEN + '/omi_document.json'))['gltf']
    keep = [nd for nd in doc['nodes'] if nd['name'] not in ('mesh', 'well', 'column', 'wind')]
    plain = dict(doc, nodes=keep)
    srv = Server(size_classes(64, per_class=2, min_bodies=32))
    req = srv.submit_document(plain, steps=90, dt=1 / 120.0)
    srv.run(clock='ticks')
    o = pyoracle.OracleWorld.from_world(gltf.build_world(plain, fixed_dt=1 / 120.0))
    for _ in range(90):
        o.step(1 / 120.0)
    st = o.state()
    n = req.world.body_count
    for col, key in zip(STATE, ('position', 'orientation', 'linear_velocity', 'angular_velocity', 'awake',
                                'sleep_timer')):
        assert np.array_equal(getattr(req.world, col)[:n], st[key]), col
    srv.close()


def test_full_class_spills_into_new_chunks_under_budget_and_waits_over_it():
    """One 2-slot class and a budget of about two and a half such arenas: the
    first chunk fills, the third request spills into a second chunk reserved
    on demand, the next reservation would pass the budget so the fifth and
    sixth requests wait for a slot to free up. Every result still equals the
    world stepped alone."""
    from omi_physics_b200.serving import SlotClass
    probe = Server([SlotClass(bodies=65, count=2)])
    one = probe.device_bytes()
    probe.close()
    srv = Server([SlotClass(bodies=65, count=2)], budget_bytes=int(2.5 * one))
    assert srv.grow
    reqs = scenes.serving_requests(6, seed=11, n_min=20, n_max=60)
    subs = []
    for i, r in enumerate(reqs):
        w, meta = scenes.serving_world(r)
        subs.append((r, srv.submit(w, 12 + i, dt=meta['dt'], arrival=0)))
    stats = srv.run(clock='ticks')
    assert stats.completed == 6
    assert stats.chunks_added == 1 and len(srv.chunks) == 2 and srv.W == 4
    assert stats.peak_active == 4                       # capacity grew past the first class
    assert sum(1 for wt in stats.wait_ms if wt > 0) == 2   # over budget: two requests waited
    assert srv.device_bytes() <= 2.5 * one
    for r, q in subs:
        w, meta = scenes.serving_world(r)
        b = WorldBatch([w], dts=[meta['dt']])
        b.step(q.steps)
        b.sync_to_host()
        for col in STATE:
            assert np.array_equal(getattr(q.world, col)[:w.body_count], getattr(w, col)[:w.body_count]), \
                (q.rid, col)
    srv.close()
