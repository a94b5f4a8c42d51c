"""Generate the golden fixtures by running the reference omi_physics itself.

Run in a container that has the reference built by ``oracle/build_ref.sh``
(into ``oracle/_ref``); the fixtures it writes are committed so the tests need
neither the reference nor its build:

    python tests/golden/make_golden.py

For each scene the fixture holds (i) the reference world's column snapshot
right after construction (``init/*``, used to check that
``omi_physics_b200.scenes`` builds identical worlds) and (ii) checkpoints: at
selected steps, every oracle input captured from the reference world (state,
tables, warm-start cache) and the reference's own results of that one step
(broadphase pairs, contacts with impulses, next-step cache, body state).
"""
import os
import sys
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle', '_ref'))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
sys.path.insert(0, ROOT)

import omi_physics as ref                       # noqa: E402  (the reference)
from omi_physics import joints as rjoints, model as rmodel   # noqa: E402
import pyoracle                                  # noqa: E402
from omi_physics_b200 import scenes              # noqa: E402

API = SimpleNamespace(PhysicsWorld=ref.PhysicsWorld, model=rmodel, joints=rjoints)

STEPS = {'pyramid': (50, (0, 3, 12, 30, 44)), 'debris': (240, (0, 90, 150, 239)),
         'convex': (180, (0, 100, 140, 179)), 'chain': (140, (0, 60, 139)),
         'spheres': (120, (0, 60, 119))}


def snapshot_init(w):
    out = {}
    n = w.body_count
    for name in (w._VEC + w._SCALAR_F + w._SCALAR_I + ('awake',)):
        out['init/' + name] = np.asarray(getattr(w, '_' + name)[:n]).copy()
    return out


def main():
    for name, (steps, checkpoints) in STEPS.items():
        w, meta = scenes.GOLDEN_SCENES[name](API)
        dt = meta['dt']
        data = snapshot_init(w)
        rec = {}
        bp = w._collision.broadphase
        orig = bp.pairs

        def recording(world, _orig=orig):
            p = _orig(world)
            rec['pairs'] = np.array(p, dtype=np.int32).reshape(-1, 2)
            return p
        bp.pairs = recording
        for s in range(steps):
            if s in checkpoints:
                ow = pyoracle.OracleWorld.from_world(w)
                for k, v in pyoracle.to_arrays(ow).items():
                    data['ck%d/in/%s' % (s, k)] = v
                rec.clear()
            w.step(dt)
            if s in checkpoints:
                p = 'ck%d/out/' % s
                cs = w.contacts
                data[p + 'pairs'] = rec.get('pairs', np.zeros((0, 2), np.int32))
                data[p + 'c_ab'] = np.array([[c.a, c.b] for c in cs], np.int32).reshape(-1, 2)
                data[p + 'c_point'] = np.array([c.point for c in cs]).reshape(-1, 3)
                data[p + 'c_normal'] = np.array([c.normal for c in cs]).reshape(-1, 3)
                data[p + 'c_depth'] = np.array([c.depth for c in cs])
                data[p + 'c_impulse'] = np.array([[c.normal_impulse, c.tangent_impulse[0],
                                                   c.tangent_impulse[1]] for c in cs]).reshape(-1, 3)
                for col in ('position', 'orientation', 'linear_velocity', 'angular_velocity',
                            'sleep_timer', 'awake', 'aabb_min', 'aabb_max'):
                    data[p + col] = np.asarray(getattr(w, col)).copy()
        data['meta/steps'] = np.array(steps)
        data['meta/checkpoints'] = np.array(checkpoints)
        data['meta/dt'] = np.array(dt)
        path = os.path.join(HERE, name + '.npz')
        np.savez_compressed(path, **data)
        print(name, 'bodies', w.body_count, 'size %.0f KB' % (os.path.getsize(path) / 1024))


if __name__ == '__main__':
    main()
