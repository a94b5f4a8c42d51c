"""The device narrowphase primitives, compiled for the host, against the
oracle and the reference's compiled primitives.

``tests/emulation/collide_host.cpp`` includes
``omi_physics_b200/csrc/geometry.cuh`` (the functions ``k_narrow`` and
``k_edge_clip`` run per pair, and the split of the box-box test between
those two kernels: face axes, then edge axes) and answers seeded box-box,
sphere-sphere and sphere-box pairs and quaternions: random poses plus the degenerate families
the step meets (aligned faces, coincident centres, exact zero-depth face
contact, quarter turns, near-parallel edges whose cross products the
separating-axis test skips, a sphere centre inside a box). Every answer
(count, normal, points, depths) must equal the oracle's bit for bit, and the
oracle's must equal the reference's compiled ``_collide_native`` functions
(``_collide_native.pyx:20-344``) and ``mathutil.quat_to_matrix``
(``mathutil.py:59-76``) when the reference is built here.
"""
import ctypes as C
import math
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import pyoracle

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), 'oracle', '_ref')
D = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(D)


@pytest.fixture(scope='module')
def emu(tmp_path_factory):
    cxx = shutil.which('g++')
    if cxx is None:
        pytest.skip('no host C++ compiler')
    out = str(tmp_path_factory.mktemp('emu') / 'libcollide_host.so')
    subprocess.run([cxx, '-O2', '-std=c++17', '-fPIC', '-shared', '-ffp-contract=off', '-o', out,
                    os.path.join(HERE, 'emulation', 'collide_host.cpp')], check=True)
    lib = C.CDLL(out)
    lib.emu_box_box.argtypes = [D] * 9
    lib.emu_box_box.restype = C.c_int
    lib.emu_box_box_split.argtypes = [D] * 9
    lib.emu_box_box_split.restype = C.c_int
    lib.emu_sphere_sphere.argtypes = [D, C.c_double, D, C.c_double, D, D, D]
    lib.emu_sphere_sphere.restype = C.c_int
    lib.emu_sphere_box.argtypes = [D, C.c_double, D, D, D, D, D, D]
    lib.emu_sphere_box.restype = C.c_int
    lib.emu_quat_to_matrix.argtypes = [D, D]
    lib.emu_quat_to_matrix.restype = None
    return lib


def _native():
    if not os.path.isdir(os.path.join(REF, 'omi_physics')):
        return None, None
    if REF not in sys.path:
        sys.path.insert(0, REF)
    from omi_physics import _collide_native, mathutil
    return _collide_native, mathutil


def _axis_quat(axis, angle):
    a = np.asarray(axis, 'd') / np.linalg.norm(axis)
    return np.array([*(a * math.sin(0.5 * angle)), math.cos(0.5 * angle)])


def _box_cases(rng, n):
    """(ca, qa, ha, cb, qb, hb) tuples: random overlapping-ish poses, then the
    degenerate families."""
    out = []
    for _ in range(n):
        ha, hb = rng.uniform(0.1, 1.0, 3), rng.uniform(0.1, 1.0, 3)
        qa, qb = rng.normal(size=4), rng.normal(size=4)
        d = rng.normal(size=3)
        d *= rng.uniform(0.0, 1.1) * (np.linalg.norm(ha) + np.linalg.norm(hb)) / np.linalg.norm(d)
        out.append((rng.normal(size=3), qa, ha, None, qb, hb, d))
    ident = np.array([0.0, 0.0, 0.0, 1.0])
    quarter = _axis_quat((0, 1, 0), 0.5 * math.pi)
    for k in range(n // 10):
        ha, hb = rng.uniform(0.2, 1.0, 3), rng.uniform(0.2, 1.0, 3)
        kind = k % 6
        if kind == 0:                                    # aligned, random offset
            out.append((np.zeros(3), ident, ha, None, ident, hb, rng.uniform(-1.0, 1.0, 3)))
        elif kind == 1:                                  # coincident centres
            out.append((np.zeros(3), rng.normal(size=4), ha, None, rng.normal(size=4), hb, np.zeros(3)))
        elif kind == 2:                                  # face on face, zero depth
            off = np.array([rng.uniform(-0.2, 0.2), ha[1] + hb[1], rng.uniform(-0.2, 0.2)])
            out.append((np.zeros(3), ident, ha, None, ident, hb, off))
        elif kind == 3:                                  # a quarter turn, overlapping
            out.append((np.zeros(3), ident, ha, None, quarter, hb, rng.uniform(-0.5, 0.5, 3)))
        elif kind == 4:                                  # near-parallel edges
            tilt = _axis_quat(rng.normal(size=3), float(rng.choice([1e-12, 1e-9, 1e-6])))
            out.append((np.zeros(3), ident, ha, None, tilt, hb, rng.uniform(-0.6, 0.6, 3)))
        else:                                            # equal boxes, one turned about an axis
            q = _axis_quat(rng.normal(size=3), rng.uniform(0, 2 * math.pi))
            out.append((np.zeros(3), ident, ha, None, q, ha.copy(), rng.uniform(-0.8, 0.8, 3)))
    return out


def _mat(lib, q):
    q = np.ascontiguousarray(q, 'd')
    R = np.zeros(9)
    lib(_p(q), _p(R))
    return R


def _box_pair(fn, ca, Ra, ha, cb, Rb, hb):
    nrm, pts, dep = np.zeros(3), np.zeros(12), np.zeros(4)
    args = [np.ascontiguousarray(x, 'd') for x in (ca, Ra, ha, cb, Rb, hb)]
    n = fn(*[_p(a) for a in args], _p(nrm), _p(pts), _p(dep))
    return n, nrm, pts[:3 * n].reshape(-1, 3), dep[:n]


def test_quaternions(emu):
    rng = np.random.default_rng(1)
    native, mathutil = _native()
    ol = pyoracle.lib()
    qs = np.concatenate([rng.normal(size=(4000, 3 + 1)) * np.exp2(rng.integers(-8, 8, (4000, 1))),
                         np.eye(4), -np.eye(4)])
    for q in qs:
        got = _mat(emu.emu_quat_to_matrix, q)
        want = _mat(ol.or_quat_to_matrix, q)
        assert np.array_equal(got, want), q
        if mathutil is not None:
            assert np.array_equal(want, mathutil.quat_to_matrix(np.asarray(q, 'd')).reshape(9)), q


def test_box_box(emu):
    rng = np.random.default_rng(2)
    native, _ = _native()
    ol = pyoracle.lib()
    hits = 0
    for ca, qa, ha, _, qb, hb, d in _box_cases(rng, 20000):
        Ra = _mat(ol.or_quat_to_matrix, qa)
        Rb = _mat(ol.or_quat_to_matrix, qb)
        cb = ca + d
        g = _box_pair(emu.emu_box_box, ca, Ra, ha, cb, Rb, hb)
        s = _box_pair(emu.emu_box_box_split, ca, Ra, ha, cb, Rb, hb)   # the step's two-kernel form
        o = _box_pair(ol.or_box_box, ca, Ra, ha, cb, Rb, hb)
        assert g[0] == o[0] and s[0] == o[0], (ca, qa, ha, cb, qb, hb)
        if o[0]:
            hits += 1
            for x, y, z in zip(g[1:], s[1:], o[1:]):
                assert np.array_equal(x, z) and np.array_equal(y, z), (ca, qa, ha, cb, qb, hb)
        if native is not None:
            n, nrm, pts, dep = native.box_box(ca, Ra.reshape(3, 3), ha, cb, Rb.reshape(3, 3), hb)
            assert n == o[0], (ca, qa, ha, cb, qb, hb)
            if n:
                assert np.array_equal(np.array(nrm), o[1])
                assert np.array_equal(np.array(pts, 'd').reshape(-1, 3), o[2])
                assert np.array_equal(np.array(dep, 'd'), o[3])
    assert hits > 5000


def test_spheres(emu):
    rng = np.random.default_rng(3)
    native, _ = _native()
    ol = pyoracle.lib()

    def run(fn, *args):
        nrm, pts, dep = np.zeros(3), np.zeros(3), np.zeros(1)
        n = fn(*args, _p(nrm), _p(pts), _p(dep))
        return n, nrm, pts, dep

    hits = 0
    for k in range(20000):
        ca = rng.normal(size=3)
        ra, rb = float(rng.uniform(0.1, 1.0)), float(rng.uniform(0.1, 1.0))
        d = rng.normal(size=3)
        d *= rng.uniform(0.0, 1.2) * (ra + rb) / np.linalg.norm(d)
        if k % 50 == 0:
            d[:] = 0.0                                   # coincident centres
        cb = ca + d
        g = run(emu.emu_sphere_sphere, _p(ca), ra, _p(cb), rb)
        o = run(ol.or_sphere_sphere, _p(ca), ra, _p(cb), rb)
        assert g[0] == o[0] and all(np.array_equal(x, y) for x, y in zip(g[1:], o[1:])) if o[0] else g[0] == 0
        if native is not None:
            n, nrm, pts, dep = native.sphere_sphere(ca, ra, cb, rb)
            assert n == o[0]
            if n:
                assert np.array_equal(np.array(nrm), o[1]) and np.array_equal(np.array(pts[0]), o[2])
                assert dep[0] == o[3][0]
        hits += o[0]
        hb = rng.uniform(0.1, 1.0, 3)
        Rb = _mat(ol.or_quat_to_matrix, rng.normal(size=4))
        cs = cb + rng.uniform(-1.0, 1.0, 3) * (hb + ra)
        if k % 50 == 1:
            cs = cb.copy()                               # centre inside the box
        g = run(emu.emu_sphere_box, _p(cs), ra, _p(cb), _p(Rb), _p(hb))
        o = run(ol.or_sphere_box, _p(cs), ra, _p(cb), _p(Rb), _p(hb))
        assert g[0] == o[0] and all(np.array_equal(x, y) for x, y in zip(g[1:], o[1:])) if o[0] else g[0] == 0
        if native is not None:
            n, nrm, pts, dep = native.sphere_box(cs, ra, cb, Rb.reshape(3, 3), hb)
            assert n == o[0]
            if n:
                assert np.array_equal(np.array(nrm), o[1]) and np.array_equal(np.array(pts[0]), o[2])
                assert dep[0] == o[3][0]
        hits += o[0]
    assert hits > 5000
