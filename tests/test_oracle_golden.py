"""Pin the C oracle to the reference: replay each golden checkpoint (the
reference's own inputs and one-step outputs) through ``or_step``.

Box/sphere/convex scenes must agree bit-for-bit: the oracle restates the
reference's arithmetic in its own order (Cython C code, numpy einsum and BLAS
FMA chains measured on numpy 2.3.5). Joints agree to 1e-12 relative: the
reference solves the 3x3 point-joint system with LAPACK dgesv, which the
oracle restates as partial-pivot LU (same result to ~1e-15).
"""
import numpy as np
import pytest

import pyoracle
from golden_util import SCENES, checkpoint, checkpoints, events_from_overlaps, load, pair_set

EXACT = ('pyramid', 'debris', 'convex', 'spheres', 'capsules', 'zones', 'terrain', 'ridge', 'conveyor',
         'degenerate', 'rods', 'convex_late')


def _close(a, b, exact):
    if exact:
        return np.array_equal(a, b)
    scale = max(1.0, float(np.max(np.abs(b))) if b.size else 1.0)
    return a.shape == b.shape and float(np.max(np.abs(a - b), initial=0.0)) <= 1e-12 * scale


@pytest.mark.parametrize('scene', SCENES)
def test_oracle_matches_reference_checkpoints(scene):
    data = load(scene)
    exact = scene in EXACT
    dt = float(data['meta/dt'])
    for step in checkpoints(data):
        ins, outs = checkpoint(data, step)
        ow = pyoracle.from_arrays(ins)
        ow.step(dt)
        assert np.array_equal(ow.pairs(), outs['pairs']), (scene, step, 'pairs')
        c = ow.contacts()
        assert np.array_equal(np.stack([c['a'], c['b']], 1).reshape(-1, 2), outs['c_ab']), (scene, step)
        for key, ref in (('point', outs['c_point']), ('normal', outs['c_normal']),
                         ('depth', outs['c_depth']), ('impulse', outs['c_impulse'])):
            assert _close(c[key].reshape(ref.shape), ref, exact), (scene, step, key)
        st = ow.state()
        for key in ('position', 'orientation', 'linear_velocity', 'angular_velocity',
                    'sleep_timer', 'aabb_min', 'aabb_max'):
            assert _close(st[key], outs[key], exact), (scene, step, key)
        assert np.array_equal(st['awake'], outs['awake']), (scene, step, 'awake')
        if 'overlaps' in outs:
            new = ow.overlaps()
            assert new == pair_set(outs['overlaps']), (scene, step, 'trigger overlaps')
            ev = events_from_overlaps(pair_set(ins['overlaps_prev']), new)
            assert np.array_equal(ev, outs['events']), (scene, step, 'trigger events')


def test_golden_scenes_exercise_every_narrowphase_route():
    """The fixtures cover box-box, sphere-sphere, sphere-box and GJK/EPA pairs
    (convex hulls and capsules / cylinders)."""
    seen = set()
    for scene in SCENES:
        data = load(scene)
        for step in checkpoints(data):
            ins, outs = checkpoint(data, step)
            kinds = ins['shape_type'][ins['collider_shape']]
            for a, b in outs['c_ab']:
                seen.add(tuple(sorted((int(kinds[a]), int(kinds[b])))))
    assert {(2, 2), (1, 1), (1, 2)} <= seen
    assert any(3 in k for k in seen)
    assert {(1, 4), (2, 4), (4, 4)} <= seen
    assert {(4, 5), (2, 5), (1, 5), (3, 5)} <= seen     # every proxy kind against a triangle mesh


def test_zones_fixture_exercises_triggers_and_volumes():
    """Sensors enter, stay and exit; all four volume behaviours are present."""
    data = load('zones')
    kinds = set()
    for step in checkpoints(data):
        ins, outs = checkpoint(data, step)
        kinds |= set(int(k) for k in outs['events'][:, 0])
        assert len(outs['overlaps']) > 5
    assert {0, 1} <= kinds
    vk = data['ck0/in/vol_kind']
    assert int(data['ck0/in/s_n_volumes']) == 4
    assert any(k & 1 for k in vk) and any(k & 8 for k in vk) and any(k & 16 for k in vk)
