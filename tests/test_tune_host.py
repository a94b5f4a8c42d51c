"""The autotuner's search and cache on the CPU, against a fake timer.

The step's launch configuration changes only speed, never results, so the
search is a plain minimisation: coordinate descent from the defaults, one
parameter at a time, each configuration measured once, with a margin that
keeps noise from moving the choice. Entries are cached per (GPU, workload
signature); the user cache wins over the shipped one.
"""
import json

import pytest

from omi_physics_b200 import scenes, tune
from omi_physics_b200._lib import DEFAULT_TUNING


def fake_timer(best, noise=None):
    """Time grows with each parameter's distance (in list position) from ``best``."""
    calls = []

    def measure(cfg):
        calls.append(dict(cfg))
        t = 1.0
        for k, v in cfg.items():
            t += 0.1 * abs(tune.SPACE[k].index(v) - tune.SPACE[k].index(best[k]))
        if noise:
            t += noise(len(calls))
        return t
    return measure, calls


def test_coordinate_search_finds_the_separable_optimum():
    best = dict(sweep_warps=4, sweep_max_split=1, pair_block=512, pair_blocks_per_sm=8,
                narrow_block=64, gjk_warps=8, wide_sweep_blocks=16, wide_cluster=8, sweep_claim=8)
    measure, calls = fake_timer(best)
    cfg, t, trials = tune.coordinate_search(measure, tune.SPACE, dict(DEFAULT_TUNING))
    assert cfg == best
    assert t == pytest.approx(1.0)
    assert trials == len(calls) == len({tuple(sorted(c.items())) for c in calls})   # memoised


def test_coordinate_search_keeps_the_default_when_nothing_beats_it_by_the_margin():
    measure, _ = fake_timer(dict(DEFAULT_TUNING), noise=lambda i: 0.0 if i == 1 else -0.005)
    cfg, _, _ = tune.coordinate_search(measure, tune.SPACE, dict(DEFAULT_TUNING), margin=0.01)
    assert cfg == DEFAULT_TUNING


def test_signature_separates_workloads():
    pyr, _ = scenes.pyramid()
    deb, _ = scenes.debris(n=300, seed=1)
    hull, _ = scenes.convex_pile(n=60, seed=1, arena=8.0, height=4.0)
    chain, _ = scenes.joint_chain(links=8, loose=8)
    sigs = {tune.signature([pyr]), tune.signature([deb]), tune.signature([hull]), tune.signature([chain]),
            tune.signature([deb] * 8)}
    assert len(sigs) == 5
    assert tune.signature([hull]).endswith('-gjk') and tune.signature([chain]).endswith('-joints')


def test_cache_store_lookup_and_precedence(tmp_path, monkeypatch):
    user = tmp_path / 'user.json'
    shipped = tmp_path / 'shipped.json'
    monkeypatch.setenv('OMI_TUNING_CACHE', str(user))
    monkeypatch.setattr(tune, 'SHIPPED', str(shipped))
    assert tune.lookup('GPU X', 'w0-n6-max6') is None
    shipped.write_text(json.dumps({'GPU X': {'w0-n6-max6': {'groups': 2, 'launch': {'pair_block': 128}}}}))
    assert tune.lookup('GPU X', 'w0-n6-max6')['groups'] == 2
    tune.store('GPU X', 'w0-n6-max6', {'groups': 3, 'launch': {}})
    assert tune.lookup('GPU X', 'w0-n6-max6')['groups'] == 3          # the user cache first
    assert tune.lookup('GPU Y', 'w0-n6-max6') is None
    tune.store('GPU X', 'other', {'groups': 1, 'launch': {}})
    data = json.loads(user.read_text())
    assert set(data['GPU X']) == {'w0-n6-max6', 'other'}
