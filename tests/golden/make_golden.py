"""Generate the golden fixtures by running the reference omi_physics itself.

Run in a container that has the reference built by ``oracle/build_ref.sh``
(into ``oracle/_ref``); the fixtures it writes are committed so the tests need
neither the reference nor its build:

    python tests/golden/make_golden.py [scene ...]

``capsule_triangles.npz`` holds capsule queries against triangle batches and
the reference's compiled ``capsule_triangles`` answers (the scene name
``capsule_triangles`` makes only that file); ``omi_document.json`` an OMI glTF
physics document with the reference's export of it (name ``omi_document``).

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
from omi_physics import omi_gltf as rgltf        # noqa: E402
import pyoracle                                  # noqa: E402
from omi_physics_b200 import scenes              # noqa: E402

API = SimpleNamespace(PhysicsWorld=ref.PhysicsWorld, model=rmodel, joints=rjoints, gravity=rgravity)
EVENT_CODES = {'enter': 0, 'stay': 1, 'exit': 2}

STEPS = {'pyramid': (50, (0, 3, 12, 30, 44)), 'debris': (240, (0, 90, 150, 239)),
         'convex': (180, (0, 100, 140, 179)), 'chain': (140, (0, 60, 139)),
         'spheres': (120, (0, 60, 119)), 'capsules': (180, (0, 40, 100, 179)),
         'zones': (150, (0, 40, 90, 149)), 'terrain': (200, (0, 100, 160, 199)),
         'ridge': (150, (0, 70, 149)), 'conveyor': (150, (0, 70, 149)),
         'degenerate': (300, (0, 1, 30, 118, 125, 250, 299)), 'rods': (240, (0, 1, 60, 150, 239)),
         'convex_late': (300, (220, 280, 299))}


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


def omi_document(seed=3, n=40):
    """An OMI glTF physics document: every shape kind, materials with combine
    modes, collision filters, a joint table, global gravity, dynamic / static /
    kinematic bodies, sensors and gravity-volume nodes (some bounded by their
    own sensor shape)."""
    rng = np.random.default_rng(seed)
    shapes = [{'type': 'box', 'box': {'size': [20.0, 1.0, 20.0]}},
              {'type': 'sphere', 'sphere': {'radius': 2.5}},
              {'type': 'box', 'box': {'size': [3.0, 4.0, 3.0]}},
              {'type': 'cylinder', 'cylinder': {'height': 1.2, 'radiusBottom': 0.3, 'radiusTop': 0.3}},
              {'type': 'trimesh', 'trimesh': {'mesh': 1}}]
    for _ in range(6):
        k = rng.integers(3)
        if k == 0:
            shapes.append({'type': 'box', 'box': {'size': [float(x) for x in rng.uniform(0.4, 1.2, 3)]}})
        elif k == 1:
            shapes.append({'type': 'sphere', 'sphere': {'radius': float(rng.uniform(0.2, 0.6))}})
        else:
            shapes.append({'type': 'capsule', 'capsule': {'height': float(rng.uniform(0.3, 1.0)),
                                                          'radius': float(rng.uniform(0.2, 0.4))}})
    mats = [{'staticFriction': 0.6, 'dynamicFriction': 0.5, 'restitution': 0.1, 'frictionCombine': 'average',
             'restitutionCombine': 'maximum'},
            {'staticFriction': 0.9, 'dynamicFriction': 0.8, 'restitution': 0.4, 'frictionCombine': 'minimum',
             'restitutionCombine': 'multiply'}]
    filters = [{'collisionSystems': ['props'], 'notCollideWithSystems': ['fx']},
               {'collisionSystems': ['fx'], 'collideWithSystems': ['ground']}]
    joints = [{'limits': [{'linearAxes': [0, 1, 2], 'min': 0.0, 'max': 0.0}, {'angularAxes': [0, 2]}],
               'drives': [{'type': 'angular', 'mode': 'force', 'axis': 1, 'velocityTarget': 2.0,
                           'maxForce': 40.0}]}]
    motion = lambda t, **kw: dict({'type': t, 'mass': 1.0, 'centerOfMass': [0, 0, 0],
                                   'inertiaDiagonal': [0, 0, 0], 'inertiaOrientation': [0, 0, 0, 1],
                                   'linearVelocity': [0, 0, 0], 'angularVelocity': [0, 0, 0],
                                   'gravityFactor': 1.0}, **kw)
    nodes = [{'name': 'ground', 'translation': [0.0, -0.5, 0.0],
              'extensions': {'OMI_physics_body': {'motion': motion('static'),
                                                  'collider': {'shape': 0, 'physicsMaterial': 0}}}},
             {'name': 'well', 'translation': [3.0, 4.0, -2.0],
              'extensions': {'OMI_physics_body': {'trigger': {'shape': 1}},
                             'OMI_physics_gravity': {'type': 'point', 'gravity': 5.0, 'priority': 2,
                                                     'replace': False, 'stop': False,
                                                     'center': [3.0, 4.0, -2.0]}}},
             {'name': 'column', 'translation': [-3.0, 2.0, 2.0],
              'extensions': {'OMI_physics_body': {'trigger': {'shape': 2}},
                             'OMI_physics_gravity': {'type': 'directional', 'gravity': 3.0, 'priority': 3,
                                                     'replace': True, 'stop': False,
                                                     'direction': [0.0, 1.0, 0.0]}}},
             {'name': 'wind', 'extensions': {'OMI_physics_gravity': {
                 'type': 'directional', 'gravity': 0.4, 'priority': 0, 'replace': False, 'stop': False,
                 'direction': [1.0, 0.0, 0.0]}}},
             {'name': 'lift', 'translation': [0.0, 0.3, 4.0], 'rotation': [0.0, 0.38268343, 0.0, 0.92387953],
              'extensions': {'OMI_physics_body': {
                  'motion': motion('kinematic', linearVelocity=[0.0, 0.0, -0.5]),
                  'collider': {'shape': 3}, 'joint': {'joint': 0, 'connectedNode': 0,
                                                      'enableCollision': True}}}},
             {'name': 'mesh', 'translation': [0.0, 0.0, 0.0],
              'extensions': {'OMI_physics_body': {'collider': {'shape': 4}}}}]
    for i in range(n):
        axis = rng.normal(size=3)
        axis /= np.linalg.norm(axis)
        ang = rng.uniform(0, np.pi)
        q = [float(x) for x in np.concatenate([axis * np.sin(ang / 2), [np.cos(ang / 2)]])]
        body = {'motion': motion('dynamic', mass=float(rng.uniform(0.5, 4.0)),
                                 linearVelocity=[float(x) for x in rng.normal(0, 0.5, 3)],
                                 gravityFactor=float(rng.uniform(0.5, 1.5))),
                'collider': {'shape': int(rng.integers(5, len(shapes)))}}
        if i % 3 == 0:
            body['collider']['physicsMaterial'] = int(rng.integers(2))
        if i % 5 == 0:
            body['collider']['collisionFilter'] = int(rng.integers(2))
        nodes.append({'name': 'item%d' % i, 'translation': [float(x) for x in rng.uniform((-4, 1, -4), (4, 6, 4))],
                      'rotation': q, 'extensions': {'OMI_physics_body': body}})
    return {'asset': {'version': '2.0'}, 'extensionsUsed': list(rgltf.SUPPORTED),
            'extensions': {'OMI_physics_shape': {'shapes': shapes},
                           'OMI_physics_body': {'physicsMaterials': mats, 'collisionFilters': filters},
                           'OMI_physics_joint': {'physicsJoints': joints},
                           'OMI_physics_gravity': {'gravity': 9.81, 'direction': [0.0, -1.0, 0.0]}},
            'nodes': nodes}


def make_omi_document():
    """tests/golden/omi_document.json: the document, the reference's own
    export of it (omi_gltf.load_document + export_extensions) and the column
    snapshot of the world built from it with the reference's classes (the
    triangle-mesh node left out)."""
    import json
    from omi_physics_b200.gltf import build_world
    gltf = omi_document()
    top, nodes = rgltf.export_extensions(rgltf.load_document(gltf))
    plain = dict(gltf, nodes=[nd for nd in gltf['nodes'] if nd['name'] != 'mesh'])
    w = build_world(plain, api=API, fixed_dt=1.0 / 120.0)
    init = {k[len('init/'):]: v.tolist() for k, v in snapshot_init(w).items()}
    out = {'gltf': gltf, 'export_top': top, 'export_nodes': {str(k): v for k, v in nodes.items()},
           'world_init': init, 'volumes': len(w.gravity_volumes)}
    path = os.path.join(HERE, 'omi_document.json')
    with open(path, 'w') as f:
        json.dump(out, f, indent=1, allow_nan=True)
    print('omi_document', len(gltf['nodes']), 'nodes', w.body_count, 'bodies')


def main(names=()):
    if not names or 'omi_document' in names:
        make_omi_document()
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
