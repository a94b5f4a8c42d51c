"""Generate the golden fixtures by running the reference omi_physics itself.

Run in a container that has the reference built by ``oracle/build_ref.sh``
(into ``oracle/_ref``); the fixtures it writes are committed so the tests need
neither the reference nor its build:

    python tests/golden/make_golden.py [scene ...]

``capsule_triangles.npz`` holds capsule queries against triangle batches and
the reference's compiled ``capsule_triangles`` answers (the scene name
``capsule_triangles`` makes only that file).

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
from omi_physics import gravity as rgravity, joints as rjoints, model as rmodel   # noqa: E402
import pyoracle                                  # noqa: E402
from omi_physics_b200 import scenes              # noqa: E402

API = SimpleNamespace(PhysicsWorld=ref.PhysicsWorld, model=rmodel, joints=rjoints, gravity=rgravity)
EVENT_CODES = {'enter': 0, 'stay': 1, 'exit': 2}

STEPS = {'pyramid': (50, (0, 3, 12, 30, 44)), 'debris': (240, (0, 90, 150, 239)),
         'convex': (180, (0, 100, 140, 179)), 'chain': (140, (0, 60, 139)),
         'spheres': (120, (0, 60, 119)), 'capsules': (180, (0, 40, 100, 179)),
         'zones': (150, (0, 40, 90, 149))}


def _pairs_array(pairs):
    return np.array(sorted(pairs), dtype=np.int32).reshape(-1, 2)


def snapshot_init(w):
    out = {}
    n = w.body_count
    for name in (w._VEC + w._SCALAR_F + w._SCALAR_I + ('awake',)):
        out['init/' + name] = np.asarray(getattr(w, '_' + name)[:n]).copy()
    return out


def _rot(axis, angle):
    a = np.asarray(axis, 'd') / np.linalg.norm(axis)
    k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(angle) * k + (1 - np.cos(angle)) * (k @ k)


def capsule_triangle_cases():
    """Capsule queries for the reference's ``capsule_triangle_batch``:
    ``[(CapsuleProxy, verts (T,3,3)), ...]``. Hand-placed floors, walls,
    ceilings, rims and slivers (the geometry of the reference's own batch
    tests), seeded random triangles around tilted capsules, degenerate
    triangles, and the candidates a grid mesh gives for a capsule resting on it."""
    from omi_physics.body import CapsuleProxy, TriangleMeshProxy
    floor = ((-10.0, 0.0, -10.0), (10.0, 0.0, -10.0), (0.0, 0.0, 10.0))
    wall = ((1.0, -10.0, -10.0), (1.0, -10.0, 10.0), (1.0, 10.0, 0.0))
    ceiling = ((-10.0, 0.0, -10.0), (0.0, 0.0, 10.0), (10.0, 0.0, -10.0))
    small = ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0))
    sliver = ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (2.0, 0.0, 0.0))
    far = ((100.0, 0.0, 100.0), (101.0, 0.0, 100.0), (100.0, 0.0, 101.0))
    cap = lambda c, half=0.5, r=0.4, R=None: CapsuleProxy(np.array(c, 'd'), half, r,
                                                          np.eye(3) if R is None else R)
    cases = []
    for c in ((0.0, 0.7, 0.0), (0.0, 1.0, 0.0), (0.0, -0.3, 0.0), (0.0, -1.0, 0.0)):
        cases.append((cap(c), np.array([floor, far, ceiling])))
    cases.append((cap((0.0, -0.7, 0.0)), np.array([ceiling])))
    cases.append((cap((0.75, 0.0, 0.0)), np.array([wall])))
    cases.append((cap((-0.2, 0.0, -0.2), 0.01), np.array([small])))
    cases.append((cap((0.5, 0.0, 0.0), 0.01), np.array([sliver, small])))
    cases.append((cap((0.0, 0.3, 0.0), R=_rot((0, 0, 1), 0.6)), np.array([floor, wall])))
    cases.append((cap((0.0, 50.0, 0.0)), np.array([floor, wall])))
    rng = np.random.default_rng(2024)
    for k in range(24):
        R = _rot(rng.normal(size=3), rng.uniform(0, 2 * np.pi))
        c = cap(rng.normal(scale=0.8, size=3), float(rng.uniform(0.0, 0.8)),
                float(rng.uniform(0.2, 0.9)), R)
        cases.append((c, rng.normal(scale=1.2, size=(128, 3, 3))))
    # degenerate triangles: repeated and collinear vertices, axis through a face
    d = rng.normal(size=(64, 3))
    degen = np.stack([np.stack([d[i], d[i], d[(i + 1) % 64]]) for i in range(32)] +
                     [np.stack([d[i], 0.5 * (d[i] + d[i + 1]), d[i + 1]]) for i in range(32)])
    cases.append((cap((0.0, 0.0, 0.0), 0.6, 0.8), degen))
    cases.append((cap((0.0, 0.0, 0.0), 0.0, 0.5), np.array([floor, small])))   # a sphere
    through = np.array([((-1.0, 0.0, -1.0), (1.0, 0.0, -1.0), (0.0, 0.0, 1.0))])
    cases.append((cap((0.0, 0.0, 0.0), 0.5, 0.3), through))
    # a grid mesh (rippled floor) and the candidates of a capsule resting on it
    cells, extent = 40, 8.0
    xs = np.linspace(-extent, extent, cells)
    pts = np.array([(x, 0.05 * np.sin(i * 0.7) * np.cos(j * 0.7), z)
                    for i, x in enumerate(xs) for j, z in enumerate(xs)], 'd')
    idx = []
    for i in range(cells - 1):
        for j in range(cells - 1):
            a, b = i * cells + j, (i + 1) * cells + j
            idx += [(a, b, a + 1), (b, b + 1, a + 1)]
    mesh = TriangleMeshProxy(pts, np.array(idx, 'i'), (0, 0, 0), np.eye(3))
    for c in ((0.0, 0.3, 0.0), (2.1, 0.5, -3.3), (-5.0, 0.9, 4.0)):
        cp = cap(c, 0.5, 0.45)
        lo, hi = cp.aabb()
        cases.append((cp, mesh.candidate_vertices(lo - 0.5, hi + 0.5)))
    return cases


def make_capsule_triangles():
    """tests/golden/capsule_triangles.npz: every case's capsule (p0, p1, r),
    triangle ranges and the reference's native batch answer."""
    from omi_physics import collide
    assert collide._native is not None, 'the reference accelerators are not built'
    caps, off, verts, hit, points, normals, depths = [], [0], [], [], [], [], []
    for cp, v in capsule_triangle_cases():
        v = np.ascontiguousarray(v, 'd').reshape(-1, 3, 3)
        h, p, nrm, dep = collide.capsule_triangle_batch(cp, v)
        caps.append(np.concatenate([cp.p0, cp.p1, [cp.radius]]))
        off.append(off[-1] + len(v))
        verts.append(v); hit.append(h); points.append(p); normals.append(nrm); depths.append(dep)
    path = os.path.join(HERE, 'capsule_triangles.npz')
    np.savez_compressed(path, caps=np.array(caps), tri_off=np.array(off, np.int64),
                        verts=np.concatenate(verts), hit=np.concatenate(hit),
                        points=np.concatenate(points), normals=np.concatenate(normals),
                        depths=np.concatenate(depths))
    print('capsule_triangles', len(caps), 'queries', off[-1], 'triangles',
          int(np.concatenate(hit).sum()), 'hits')


def main(names=()):
    if not names or 'capsule_triangles' in names:
        make_capsule_triangles()
    for name, (steps, checkpoints) in STEPS.items():
        if names and name not in names:
            continue
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
        events = []
        w.add_trigger_listener(lambda kind, t, o: events.append((EVENT_CODES[kind], t, o)))
        for s in range(steps):
            if s in checkpoints:
                ow = pyoracle.OracleWorld.from_world(w)
                for k, v in pyoracle.to_arrays(ow).items():
                    data['ck%d/in/%s' % (s, k)] = v
                data['ck%d/in/overlaps_prev' % s] = _pairs_array(w._collision.triggers.overlaps)
                rec.clear()
            events.clear()
            w.step(dt)
            if s in checkpoints:
                data['ck%d/out/overlaps' % s] = _pairs_array(w._collision.triggers.overlaps)
                data['ck%d/out/events' % s] = np.array(sorted(events), dtype=np.int32).reshape(-1, 3)
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
    main(sys.argv[1:])          # scene names; none = every scene
