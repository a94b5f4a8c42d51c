"""The wide path on the GPU: every colliding world run as a wide world.

A world above the wide threshold (3072 bodies by default) runs its sort,
sweep links, wake, contact sweep, warm-start cache store, positions and
sleep on many blocks (``csrc/wide.cuh``) instead of one block per world. The
full-size configurations exercise it (``test_gpu_configs.py``: debris 4096,
convex pile 32768); here ``OMI_WIDE_THRESHOLD=0`` makes every colliding world
wide, so the reference's golden checkpoints, the oracle trajectories, the
random fuzz worlds and the wake pass's sequential cascade all run through the
wide kernels and must match bit for bit as they do through the per-world
ones. A batch with both kinds of world checks that they share an arena.
"""
import numpy as np
import pytest

import pyoracle
import test_gpu_edges as E
import test_gpu_fuzz as F
import test_gpu_parity as P
from golden_util import SCENES
from omi_physics_b200 import WorldBatch, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def every_world_wide(monkeypatch):
    monkeypatch.setenv('OMI_WIDE_THRESHOLD', '0')


@pytest.mark.parametrize('scene', SCENES)
def test_golden_checkpoints_wide(scene):
    P.test_golden_checkpoints_on_gpu(scene)


@pytest.mark.parametrize('name,builder,steps', [
    ('pyramid', lambda: scenes.pyramid(), 120),
    ('debris512', lambda: scenes.debris(n=512, seed=1, extent=8.0, height=12.0, ground=30.0), 150),
    ('convex160', lambda: scenes.convex_pile(n=160, seed=2, arena=10.0, height=8.0), 150),
    ('zones300', lambda: scenes.zones(n=300, seed=4, extent=6.0, height=10.0), 150),
    ('terrain150', lambda: scenes.terrain(n=150, seed=2, cells=30, extent=8.0), 150),
    ('degenerate', lambda: scenes.degenerate(), 300),
])
def test_trajectory_wide(name, builder, steps):
    P.test_trajectory_matches_oracle_every_step(name, builder, steps)


def test_fuzz_worlds_wide():
    F.test_random_worlds_batched_match_the_oracle()


def test_world_switches_wide():
    F.test_world_switches_batched_match_the_oracle()


def test_empty_and_static_worlds_wide():
    E.test_empty_and_static_worlds_batched_with_degenerate_contacts()


def test_wake_cascade_wide():
    E.test_wake_cascade_from_a_moving_sleeper()


def test_wide_and_per_world_worlds_in_one_arena(monkeypatch):
    """Threshold 400: two debris worlds above it run wide, three below run one
    block each, all in one batch, every world equal to the oracle each step."""
    monkeypatch.setenv('OMI_WIDE_THRESHOLD', '400')
    built = [scenes.debris(n=n, seed=60 + n, extent=4.0 + n / 120.0, height=6.0, ground=30.0)
             for n in (90, 700, 250, 1200, 30)]
    worlds = [w for w, _ in built]
    dts = [m['dt'] for _, m in built]
    oracles = [pyoracle.OracleWorld.from_world(w) for w in worlds]
    b = WorldBatch(worlds, dts=dts)
    for s in range(100):
        b.step(1)
        b.sync_to_host()
        for i, (w, o) in enumerate(zip(worlds, oracles)):
            o.step(dts[i])
            st = o.state()
            n = w.body_count
            tag = 'world %d step %d' % (i, s)
            assert np.array_equal(b.pairs(i), o.pairs()), tag
            assert np.array_equal(b.contact_arrays(i)['impulse'], o.contacts()['impulse']), tag
            for col in ('position', 'orientation', 'linear_velocity', 'angular_velocity', 'sleep_timer'):
                assert np.array_equal(getattr(w, '_' + col)[:n], st[col]), tag + ' ' + col
            assert np.array_equal(w._awake[:n], st['awake']), tag
    assert (b.levels()[[1, 3]] < 0).all() and (b.levels()[[0, 2, 4]] >= 0).all()


@pytest.mark.parametrize('budget', [64, 1400, 0])
def test_cluster_hands_off_worlds_that_do_not_fit(budget):
    """The cluster sweep takes a wide world only while every CTA's body
    records and run tables fit its shared memory; otherwise the many-block
    sweep launched after it does. A budget of 64 ints per CTA fits no world
    (every step hands off), 1400 lies near the debris world's needs as its
    contacts grow (the form may change between steps), 0 is the whole of
    shared memory (the cluster sweeps every step). Every step matches the
    oracle bit for bit, whichever form swept it."""
    w, meta = scenes.debris(n=512, seed=1, extent=8.0, height=12.0, ground=30.0)
    dt = meta['dt']
    o = pyoracle.OracleWorld.from_world(w)
    b = WorldBatch([w], dts=[dt])
    if b.ctx.tuning()['wide_cluster'] == 0:
        pytest.skip('this GPU schedules no sweep cluster')
    b.ctx.set_cluster_budget(budget)
    forms = set()
    for s in range(150):
        b.step(1)
        b.sync_to_host()
        o.step(dt)
        P._compare_step(b, w, o, 'budget %d step %d' % (budget, s))
        forms.add(int(b.levels()[0]))
    if budget == 64:
        assert forms <= {-2, 0}
    if budget == 0:
        assert -1 in forms and -2 not in forms
    b.ctx.set_cluster_budget(0)
