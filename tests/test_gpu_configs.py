"""The workload configurations at full size, against the oracle.

* debris field, 4096 bodies (1/120 s, 8 iterations): 240 steps, compared bit
  for bit at checkpoints;
* convex-hull pile, 32768 bodies (50% boxes, 25% spheres, 25% hulls through
  GJK/EPA, walled arena): its whole 300-step run, compared bit for bit every
  50 steps. Both this world and the debris field are wide worlds (their sort,
  sweep links, wake, sweep, cache store and sleep pass on many blocks);
* capsule pile, 4096 bodies (30% capsules, 20% cylinders, the rest boxes and
  spheres): 120 steps, compared bit for bit every 40 steps;
* terrain, 2000 bodies on an 18,432-triangle static mesh: 120 steps, compared
  bit for bit every 40 steps;
* the serving mix, 1024 worlds (417K bodies) as 4 concurrent groups: 240
  steps, 40 sampled worlds bit for bit, size-independent checks on all;
* batched joint chains (point joints, motors, loose boxes; 1/240 s, 12 contact
  and 12 joint iterations): 8 worlds of uneven sizes in one batch, each within
  1e-6 m / 1e-6 of the oracle after 60 steps (point joints go through an
  explicit 3x3 solve that matches the reference's LAPACK call to ~1e-12);
  and at full size, 512 such worlds for 480 steps (16 compared at step 120,
  size-independent checks on all at 480).
"""
import numpy as np
import pytest

import pyoracle
from omi_physics_b200 import WorldBatch, scenes

pytestmark = pytest.mark.gpu

STATE = ('position', 'orientation', 'linear_velocity', 'angular_velocity', 'sleep_timer')


def _check_exact(b, i, w, o, tag):
    st = o.state()
    n = w.body_count
    assert np.array_equal(b.pairs(i), o.pairs()), tag + ' pairs'
    c, oc = b.contact_arrays(i), o.contacts()
    assert np.array_equal(c['a'], oc['a']) and np.array_equal(c['b'], oc['b']), tag + ' contacts'
    assert np.array_equal(c['impulse'], oc['impulse']), tag + ' impulses'
    for col in STATE:
        assert np.array_equal(getattr(w, '_' + col)[:n], st[col]), tag + ' ' + col
    assert np.array_equal(w._awake[:n], st['awake']), tag + ' awake'
    lab = b.islands(i)
    islands_gpu = {}
    for body, l in enumerate(lab):
        if l >= 0:
            islands_gpu.setdefault(int(l), set()).add(body)
    assert {frozenset(s) for s in islands_gpu.values()} == o.islands(), tag + ' islands'


def _run_exact(w, dt, steps, every, tag):
    o = pyoracle.OracleWorld.from_world(w)
    b = WorldBatch([w], dts=[dt])
    done = 0
    while done < steps:
        k = min(every, steps - done)
        b.step(k)
        for _ in range(k):
            o.step(dt)
        done += k
        b.sync_to_host()
        _check_exact(b, 0, w, o, '%s step %d' % (tag, done))
    return b


def test_debris_4096_full_size():
    w, meta = scenes.debris(n=4096, seed=0)
    b = _run_exact(w, meta['dt'], 240, 40, 'debris4096')
    assert b.counts()[1][0] > 1000                      # settled into contact


def test_convex_pile_32768_full_size():
    """The whole 300-step run of the configuration (a wide world: its
    per-world stages on many blocks, the sweep on a thread-block cluster),
    bit for bit against the oracle every 50 steps, sleep flags and islands
    included."""
    w, meta = scenes.convex_pile(n=32768, seed=0)
    b = _run_exact(w, meta['dt'], 300, 50, 'convex32768')
    assert b.counts()[1][0] > 10000


def test_capsule_pile_4096_full_size():
    """4096 capsules / cylinders / boxes / spheres: every capsule pair through
    GJK/EPA, 120 steps compared bit for bit every 40."""
    w, meta = scenes.capsule_pile(n=4096, seed=0)
    b = _run_exact(w, meta['dt'], 120, 40, 'capsules4096')
    assert b.counts()[1][0] > 1000


def test_terrain_2000_on_an_18k_triangle_mesh():
    """2000 capsules, boxes, spheres and hulls onto a 96x96-cell rippled mesh
    (18,432 triangles, the triangle grid's full 64-cell resolution) and a
    small ramp: 120 steps compared bit for bit every 40."""
    w, meta = scenes.terrain(n=2000, seed=5, cells=96, extent=20.0)
    b = _run_exact(w, meta['dt'], 120, 40, 'terrain2000')
    assert b.counts()[1][0] > 1000


def test_batched_joint_chains():
    rng = np.random.default_rng(5)
    worlds, dts = [], []
    for k in range(8):
        w, meta = scenes.joint_chain(links=int(rng.integers(16, 65)), loose=int(rng.integers(32, 129)),
                                     seed=100 + k)
        worlds.append(w)
        dts.append(meta['dt'])
    refs = [pyoracle.OracleWorld.from_world(w) for w in worlds]
    b = WorldBatch(worlds, dts=dts)
    b.step(60)
    b.sync_to_host()
    for k, (w, o) in enumerate(zip(worlds, refs)):
        for _ in range(60):
            o.step(dts[k])
        st = o.state()
        n = w.body_count
        assert float(np.max(np.abs(w._position[:n] - st['position']))) < 1e-6, k
        assert float(np.max(np.abs(w._orientation[:n] - st['orientation']))) < 1e-6, k
        assert np.array_equal(w._awake[:n], st['awake']), k


def test_serving_mix_1024_worlds_full_size():
    """The measured workload itself: the 1024-world serving mix (417K bodies)
    stepped as 4 concurrent groups for 240 steps (the bench's pre-roll, into the
    contact-heavy regime). A seeded sample of 40 worlds, the 8 largest among
    them, equals the oracle bit for bit (pairs, contacts, impulses, state,
    islands); every world passes size-independent checks (finite state,
    unit quaternions, sleeping dynamic bodies at rest, every pair (a < b)
    unique and within the world)."""
    from omi_physics_b200.groups import WorldGroups
    reqs = scenes.serving_requests(1024, seed=0)
    worlds, dts = [], []
    for r in reqs:
        w, meta = scenes.serving_world(r)
        worlds.append(w)
        dts.append(meta['dt'])
    sizes = np.array([w.body_count for w in worlds])
    rng = np.random.default_rng(17)
    largest = list(np.argsort(-sizes, kind='stable')[:8])
    rest = [i for i in range(len(worlds)) if i not in set(largest)]
    sample = sorted(largest + list(rng.choice(rest, size=32, replace=False)))
    oracles = {int(i): pyoracle.OracleWorld.from_world(worlds[i]) for i in sample}
    g = WorldGroups(worlds, dts=dts, groups=4)
    try:
        g.step(240)
        g.sync_to_host()
        for i, o in oracles.items():
            for _ in range(240):
                o.step(dts[i])
            b, j = g.batch_of(i)
            _check_exact(b, j, worlds[i], o, 'mix world %d (%d bodies)' % (i, sizes[i]))
        for i, w in enumerate(worlds):
            n = w.body_count
            assert np.isfinite(w._position[:n]).all() and np.isfinite(w._linear_velocity[:n]).all(), i
            qn = np.linalg.norm(w._orientation[:n], axis=1)
            assert np.all(np.abs(qn - 1.0) < 1e-9), i
            asleep = (~w._awake[:n]) & (w._motion_type[:n] == 2)
            assert not np.any(w._linear_velocity[:n][asleep]) and not np.any(w._angular_velocity[:n][asleep]), i
            p = g.pairs(i)
            if len(p):
                assert (p[:, 0] < p[:, 1]).all() and p.min() >= 0 and p.max() < n, i
                assert len({tuple(x) for x in p.tolist()}) == len(p), i
    finally:
        g.close()


def test_joint_chains_512_worlds_full_size():
    """The joints configuration at full size: 512 worlds, each a chain of
    16-128 links pinned at both ends (point joints, 10% with an angular motor)
    under 64-512 loose boxes, 1/240 s, 12 contact and 12 joint iterations,
    480 steps in one batch. The chains are chaotic: on the oracle alone a
    1e-12 m nudge of the initial poses grows past 1e-9 m by step 240 and to
    about 1 m by step 480, so 16 seeded worlds are compared with the oracle
    at step 120 (within 1e-6, point joints matching LAPACK to ~1e-12 per
    solve) and all 512 pass size-independent checks at step 480 (finite
    state, unit quaternions, sleeping dynamic bodies at rest)."""
    worlds, dts = scenes.joint_chains(512, seed=21)
    rng = np.random.default_rng(22)
    sample = sorted(int(i) for i in rng.choice(512, size=16, replace=False))
    oracles = {i: pyoracle.OracleWorld.from_world(worlds[i]) for i in sample}
    b = WorldBatch(worlds, dts=dts)
    b.step(120)
    b.sync_to_host()
    for i, o in oracles.items():
        for _ in range(120):
            o.step(dts[i])
        st = o.state()
        w = worlds[i]
        n = w.body_count
        assert float(np.max(np.abs(w._position[:n] - st['position']))) < 1e-6, i
        assert float(np.max(np.abs(w._orientation[:n] - st['orientation']))) < 1e-6, i
        assert np.array_equal(w._awake[:n], st['awake']), i
    b.step(360)
    b.sync_to_host()
    for i, w in enumerate(worlds):
        n = w.body_count
        assert np.isfinite(w._position[:n]).all() and np.isfinite(w._angular_velocity[:n]).all(), i
        assert np.all(np.abs(np.linalg.norm(w._orientation[:n], axis=1) - 1.0) < 1e-9), i
        asleep = (~w._awake[:n]) & (w._motion_type[:n] == 2)
        assert not np.any(w._linear_velocity[:n][asleep]) and not np.any(w._angular_velocity[:n][asleep]), i
