"""The device GJK/EPA code, compiled for the host, against the oracle.

``tests/emulation/gjk_host.cpp`` includes ``omi_physics_b200/csrc/gjk.cuh``
with one lane per warp (the warp-wide searches reduce to the lane's own
values) and builds the proxies as ``k_gjk`` does. Every candidate pair with a
hull or capsule along 20 oracle steps of a capsule pile and a convex pile must
give the oracle's ``or_collide_convex`` answer bit for bit: contact or not,
normal, point and depth. This checks the device's support functions and its
bounded polytope storage without a GPU.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import pyoracle
from omi_physics_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
D = C.POINTER(C.c_double)
CODES = {'sphere': 1, 'box': 2, 'convex': 3, 'capsule': 4, 'cylinder': 4}
ARGS = [C.c_int, D, D, D, C.c_double, D, C.c_int] * 2 + [D, D, D]


@pytest.fixture(scope='module')
def emu(tmp_path_factory):
    cxx = shutil.which('g++')
    if cxx is None:
        pytest.skip('no host C++ compiler')
    out = str(tmp_path_factory.mktemp('emu') / 'libgjk_host.so')
    subprocess.run([cxx, '-O2', '-std=c++17', '-fPIC', '-shared', '-ffp-contract=off', '-o', out,
                    os.path.join(HERE, 'emulation', 'gjk_host.cpp')], check=True)
    lib = C.CDLL(out)
    lib.emu_collide.argtypes = ARGS
    lib.emu_collide.restype = C.c_int
    orc = pyoracle.lib()
    orc.or_collide_convex.argtypes = ARGS
    orc.or_collide_convex.restype = C.c_int
    return lib, orc


def _body(w, i, st):
    s = w.shapes[int(w._collider_shape[i])]
    k = CODES[s.type]
    c = np.ascontiguousarray(st['position'][i])
    q = np.ascontiguousarray(st['orientation'][i])
    if k == 4:
        size, r = np.array([0.0, float(s.height), 0.0]), float(s.radiusBottom)
    else:
        size, r = (np.asarray(s.size, 'd').copy() if k == 2 else np.zeros(3)), float(s.radius)
    pts = np.ascontiguousarray(s.points, 'd') if k == 3 else np.zeros((1, 3))
    return k, c, q, size, r, pts, (len(pts) if k == 3 else 0)


@pytest.mark.parametrize('name,builder', [
    ('capsules', lambda: scenes.capsule_pile(n=600, seed=2, arena=14.0, height=10.0)),
    ('convex', lambda: scenes.convex_pile(n=600, seed=3, arena=14.0, height=10.0)),
])
def test_device_gjk_equals_oracle_pair_by_pair(emu, name, builder):
    lib, orc = emu
    p = lambda a: a.ctypes.data_as(D)
    w, meta = builder()
    o = pyoracle.OracleWorld.from_world(w)
    compared = hits = 0
    for step in range(20):
        o.step(meta['dt'])
        st = o.state()
        for a, b in o.pairs():
            A, B = _body(w, a, st), _body(w, b, st)
            if A[0] < 3 and B[0] < 3:
                continue
            got = [np.zeros(3), np.zeros(3), np.zeros(1)]
            want = [np.zeros(3), np.zeros(3), np.zeros(1)]
            rg = lib.emu_collide(A[0], p(A[1]), p(A[2]), p(A[3]), A[4], p(A[5]), A[6],
                                 B[0], p(B[1]), p(B[2]), p(B[3]), B[4], p(B[5]), B[6], *map(p, got))
            rw = orc.or_collide_convex(A[0], p(A[1]), p(A[2]), p(A[3] * 0.5), A[4], p(A[5]), A[6],
                                       B[0], p(B[1]), p(B[2]), p(B[3] * 0.5), B[4], p(B[5]), B[6],
                                       *map(p, want))
            assert rg == rw, (name, step, a, b)
            if rw > 0:
                hits += 1
                for g, x in zip(got, want):
                    assert np.array_equal(g, x), (name, step, a, b)
            compared += 1
    assert compared > 2000 and hits > 200
