"""Shared helpers: build a world from a golden checkpoint and compare results."""
import numpy as np

from golden_util import checkpoint, load
from omi_physics_b200 import scenes


def world_at_checkpoint(scene, step):
    """This package's world for a golden scene, with the checkpoint's input state.

    Returns ``(world, dt, inputs, outputs)``; the world's joint objects carry
    the checkpoint's lazily fixed joint state.
    """
    data = load(scene)
    ins, outs = checkpoint(data, step)
    w, _ = scenes.GOLDEN_SCENES[scene]()
    n = w.body_count
    assert n == int(ins['s_n'])
    w._position[:n] = ins['pos']
    w._orientation[:n] = ins['q']
    w._linear_velocity[:n] = ins['v']
    w._angular_velocity[:n] = ins['w']
    w._awake[:n] = ins['awake'].astype(bool)
    w._sleep_timer[:n] = ins['sleep_timer']
    for j, c in enumerate(w.joint_constraints):
        kind = getattr(c, 'kind', '')
        if kind == 'point':
            c.local_a = ins['j_local_a'][j].copy() if ins['j_has_local_a'][j] else None
            c.local_b = ins['j_local_b'][j].copy() if ins['j_has_local_b'][j] else None
        elif kind == 'distance':
            c.length = float(ins['j_length'][j]) if ins['j_has_length'][j] else None
        elif kind == 'motor':
            c.accum = float(ins['j_accum'][j])
    return w, float(data['meta/dt']), ins, outs


def assert_close(a, b, rel, what):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if rel == 0:
        assert np.array_equal(a, b), (what, float(np.max(np.abs(a - b), initial=0.0)))
        return
    scale = max(1.0, float(np.max(np.abs(b), initial=0.0)))
    err = float(np.max(np.abs(a - b), initial=0.0))
    assert err <= rel * scale, (what, err)
