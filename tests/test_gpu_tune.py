"""The launch configuration changes speed only: every configuration the
autotuner may pick steps the same worlds to the same bits, and the autotuner
runs end to end on the GPU and caches its choice."""
import numpy as np
import pytest

from omi_physics_b200 import WorldBatch, scenes, tune
from omi_physics_b200.groups import WorldGroups

pytestmark = pytest.mark.gpu

STATE = ('_position', '_orientation', '_linear_velocity', '_angular_velocity', '_awake', '_sleep_timer')
OTHER = dict(sweep_warps=4, sweep_max_split=1, pair_block=512, pair_blocks_per_sm=8, narrow_block=64,
             gjk_warps=8, wide_sweep_blocks=1, wide_cluster=0, sweep_claim=8)


def _worlds():
    out = [scenes.debris(n=n, seed=40 + n, extent=5.0 + n / 100.0, height=6.0, ground=30.0)
           for n in (37, 150, 600)]
    out.append(scenes.convex_pile(n=120, seed=3, arena=9.0, height=5.0))
    return [w for w, _ in out], [m['dt'] for _, m in out]


@pytest.mark.parametrize('cfg,wide', [(OTHER, None), (dict(sweep_warps=8, sweep_max_split=2, pair_block=128,
                                                          pair_blocks_per_sm=32, narrow_block=256, gjk_warps=2,
                                                          wide_sweep_blocks=5, wide_cluster=8, sweep_claim=16),
                                       None),
                                      (OTHER, '0'), (dict(OTHER, wide_sweep_blocks=7), '0'),
                                      (dict(OTHER, wide_cluster=8), '0'), (dict(OTHER, wide_cluster=16), '0')])
def test_any_launch_configuration_gives_the_same_bits(cfg, wide, monkeypatch):
    """Each configuration against the defaults, with the per-world stages
    (wide=None) and with every world wide (wide='0': one-block and
    multi-block sweeps of wide worlds)."""
    if wide is not None:
        monkeypatch.setenv('OMI_WIDE_THRESHOLD', wide)
    wa, dts = _worlds()
    wb, _ = _worlds()
    a = WorldBatch(wa, dts=dts)
    b = WorldBatch(wb, dts=dts)
    b.ctx.set_tuning(**cfg)
    assert b.ctx.tuning() == cfg
    a.step(90)
    b.step(90)
    a.sync_to_host()
    b.sync_to_host()
    for i in range(len(wa)):
        assert np.array_equal(a.pairs(i), b.pairs(i)), i
        n = wa[i].body_count
        for col in STATE:
            assert np.array_equal(getattr(wa[i], col)[:n], getattr(wb[i], col)[:n]), (i, col)


def test_autotune_runs_and_is_applied_by_default(tmp_path, monkeypatch):
    monkeypatch.setenv('OMI_TUNING_CACHE', str(tmp_path / 'tuning.json'))
    worlds, dts = _worlds()
    entry = tune.autotune(worlds, dts, steps=3, warmup=1, rounds=1, groups=(2, 1))
    assert set(entry['launch']) == set(OTHER) and entry['groups'] in (1, 2)
    assert 0 < entry['ms'] <= entry['default_ms']          # the search accepts only improvements
    assert tune.tuned_for(worlds) == entry
    g = WorldGroups(worlds, dts=dts)
    try:
        assert len(g.batches) == min(entry['groups'], len(worlds))
        for b in g.batches:
            assert b.ctx.tuning() == entry['launch']
    finally:
        g.close()
