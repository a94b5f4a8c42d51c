"""Capsule against triangles on the GPU through the C ABI.

(1) The reference's own answers (``tests/golden/capsule_triangles.npz``, made
by its compiled ``capsule_triangles``) reproduced bit for bit, in one batched
call and one call per capsule. (2) A few million seeded triangles around
thousands of capsules, several pipeline chunks, against the oracle bit for
bit. (3) The device-buffer form equals the host form. (4) Ragged and empty
inputs, and refused ranges. (5) Drop-in: the reference's mesh collisions and
its character controller run through :class:`NativeShim` and give exactly
what the compiled routine gives.
"""
import os
import sys

import numpy as np
import pytest

import pyoracle
from golden_util import GOLDEN
from omi_physics_b200 import collide as oc
from omi_physics_b200._lib import OmiError

pytestmark = pytest.mark.gpu

FIX = np.load(GOLDEN + '/capsule_triangles.npz')
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, 'oracle', '_ref')


def _same(got, hit, points, normals, depths, tag=''):
    h, p, n, d = got
    assert np.array_equal(np.asarray(h).astype(bool), np.asarray(hit).astype(bool)), tag + ' hit'
    assert np.array_equal(p, points), tag + ' points'
    assert np.array_equal(n, normals), tag + ' normals'
    assert np.array_equal(d, depths), tag + ' depths'


def test_reference_answers_in_one_batched_call():
    got = oc.capsule_triangles_many(FIX['caps'], FIX['tri_off'], FIX['verts'])
    _same(got, FIX['hit'], FIX['points'], FIX['normals'], FIX['depths'])


def test_reference_answers_one_capsule_per_call():
    off = FIX['tri_off']
    for q, c in enumerate(FIX['caps']):
        s, e = int(off[q]), int(off[q + 1])
        cap = type('Cap', (), {})()
        cap.p0, cap.p1, cap.radius = c[:3], c[3:6], c[6]
        got = oc.capsule_triangle_batch(cap, FIX['verts'][s:e])
        _same(got, FIX['hit'][s:e], FIX['points'][s:e], FIX['normals'][s:e], FIX['depths'][s:e], str(q))


def _random_batch(q, seed, lo=1, hi=512):
    rng = np.random.default_rng(seed)
    counts = rng.integers(lo, hi, size=q)
    counts[::97] = 0                                     # capsules with no candidates
    centres = rng.uniform(-50, 50, size=(q, 3))
    axes = rng.normal(size=(q, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    half = rng.uniform(0.0, 0.9, size=q)
    caps = np.concatenate([centres - axes * half[:, None], centres + axes * half[:, None],
                           rng.uniform(0.2, 0.8, size=(q, 1))], axis=1)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    owner = np.repeat(np.arange(q), counts)
    verts = centres[owner][:, None, :] + rng.normal(scale=1.0, size=(len(owner), 3, 3))
    return caps, off, verts


def test_millions_of_triangles_match_the_oracle_across_chunks():
    caps, off, verts = _random_batch(18000, seed=7)
    n = len(verts)
    assert n > 4_000_000                                 # three pipeline chunks
    got = oc.capsule_triangles_many(caps, off, verts)
    hit = np.zeros(n, bool)
    pts, nrm, dep = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
    for q in range(len(caps)):
        s, e = int(off[q]), int(off[q + 1])
        if e > s:
            hit[s:e], pts[s:e], nrm[s:e], dep[s:e] = pyoracle.capsule_triangles(
                caps[q, :3], caps[q, 3:6], caps[q, 6], verts[s:e])
    assert 0.05 < hit.mean() < 0.95
    _same(got, hit, pts, nrm, dep)


def test_device_buffers_give_the_host_answer():
    import torch
    caps, off, verts = _random_batch(3000, seed=11)
    n = len(verts)
    want = oc.capsule_triangles_many(caps, off, verts)
    dev = torch.device('cuda', 0)
    tc = torch.from_numpy(caps).to(dev)
    to = torch.from_numpy(off).to(dev)
    tv = torch.from_numpy(verts).to(dev)
    th = torch.full((n,), 7, dtype=torch.uint8, device=dev)
    tp = torch.full((n, 3), 9.0, dtype=torch.float64, device=dev)
    tn = torch.full((n, 3), 9.0, dtype=torch.float64, device=dev)
    td = torch.full((n,), 9.0, dtype=torch.float64, device=dev)
    ctx, lock = oc.context(0)
    with lock:
        ctx.call('set_stream', torch.cuda.current_stream(dev).cuda_stream)
        oc.capsule_triangles_device(ctx, len(caps), tc.data_ptr(), to.data_ptr(), tv.data_ptr(), n,
                                    th.data_ptr(), tp.data_ptr(), tn.data_ptr(), td.data_ptr())
        torch.cuda.synchronize(dev)
        ctx.call('set_stream', None)
    _same((th.cpu().numpy(), tp.cpu().numpy(), tn.cpu().numpy(), td.cpu().numpy()), *want)


def test_empty_and_ragged_inputs():
    h, p, n, d = oc.capsule_triangles_many(np.zeros((2, 7)), np.zeros(3, np.int64), np.zeros((0, 3, 3)))
    assert len(h) == len(p) == len(n) == len(d) == 0
    caps, off, verts = _random_batch(5, seed=3, lo=0, hi=3)   # some capsules own nothing
    got = oc.capsule_triangles_many(caps, off, verts)
    for q in range(5):
        s, e = int(off[q]), int(off[q + 1])
        if e > s:
            want = pyoracle.capsule_triangles(caps[q, :3], caps[q, 3:6], caps[q, 6], verts[s:e])
            _same(tuple(g[s:e] for g in got), *want, tag=str(q))


def test_bad_ranges_are_refused():
    caps, off, verts = _random_batch(4, seed=5, lo=2, hi=5)
    bad = off.copy()
    bad[-1] += 1                                       # does not end at n
    with pytest.raises(OmiError):
        oc.capsule_triangles_many(caps, bad, verts)
    bad = off.copy()
    bad[1], bad[2] = bad[2], bad[1] - 1                # decreasing
    with pytest.raises(OmiError):
        oc.capsule_triangles_many(caps, bad, verts)


def _reference():
    if not os.path.isdir(os.path.join(REF, 'omi_physics')):
        pytest.skip('the reference is not built (oracle/build_ref.sh)')
    if REF not in sys.path:
        sys.path.insert(0, REF)
    from omi_physics import collide
    if collide._native is None:
        pytest.skip('the reference accelerators are not built')
    return collide


def _grid_mesh(cells=40, extent=8.0):
    from omi_physics.body import TriangleMeshProxy
    xs = np.linspace(-extent, extent, cells)
    pts = np.array([(x, 0.05 * np.sin(i * 0.7) * np.cos(j * 0.7), z)
                    for i, x in enumerate(xs) for j, z in enumerate(xs)], 'd')
    idx = []
    for i in range(cells - 1):
        for j in range(cells - 1):
            a, b = i * cells + j, (i + 1) * cells + j
            idx += [(a, b, a + 1), (b, b + 1, a + 1)]
    return pts, np.array(idx, 'i'), TriangleMeshProxy(pts, np.array(idx, 'i'), (0, 0, 0), np.eye(3))


def test_reference_mesh_collisions_through_the_shim():
    collide = _reference()
    from omi_physics.body import CapsuleProxy
    _pts, _idx, mesh = _grid_mesh()
    rng = np.random.default_rng(1)
    native = collide._native
    for k in range(12):
        cap = CapsuleProxy(np.array([rng.uniform(-6, 6), rng.uniform(0.1, 1.0), rng.uniform(-6, 6)]),
                           0.5, 0.45, np.eye(3))
        want_c = collide.collide(0, 1, cap, mesh)
        want_p = collide.capsule_mesh_pushes(cap, mesh)
        collide._native = oc.NativeShim(native)
        try:
            got_c = collide.collide(0, 1, cap, mesh)
            got_p = collide.capsule_mesh_pushes(cap, mesh)
        finally:
            collide._native = native
        assert len(got_c) == len(want_c)
        for a, b in zip(got_c, want_c):
            assert (a.a, a.b) == (b.a, b.b) and a.depth == b.depth
            assert np.array_equal(a.point, b.point) and np.array_equal(a.normal, b.normal)
        assert np.array_equal(got_p[0], want_p[0]) and np.array_equal(got_p[1], want_p[1])


def test_reference_character_controllers_walk_identically_through_the_shim():
    collide = _reference()
    from omi_physics import model
    from omi_physics.character import CharacterCapabilities, CharacterController
    from omi_physics.world import PhysicsWorld
    pts, idx, _mesh = _grid_mesh(cells=30, extent=12.0)

    def walk():
        world = PhysicsWorld(gravity=model.Gravity(gravity=9.81, direction=(0, -1, 0)))
        shape = world.add_shape(model.Shape.trimesh(points=pts, indices=idx))
        world.add_body(model.Motion(type=model.STATIC), collider=model.Collider(shape=shape),
                       position=(0, 0, 0))
        rng = np.random.default_rng(4)
        walkers = []
        for _ in range(8):
            x, z = rng.uniform(-8.0, 8.0, size=2)
            c = CharacterController(world, CharacterCapabilities(), (x, 1.2, z))
            c.safe_bind((x, 1.2, z))
            c.set_move(np.array([1.0, 0.0, 0.3]))
            walkers.append(c)
        for _ in range(20):
            for c in walkers:
                c.update(1 / 60.0)
        return np.array([c.position for c in walkers])

    want = walk()
    native = collide._native
    collide._native = oc.NativeShim(native)
    try:
        got = walk()
    finally:
        collide._native = native
    assert np.array_equal(got, want)
