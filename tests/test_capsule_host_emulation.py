"""The device capsule-against-triangle arithmetic, compiled for the host,
against the oracle and the reference's answers.

``tests/emulation/capsule_host.cpp`` includes
``omi_physics_b200/csrc/capsule.cuh`` (the per-triangle device function the
kernel runs, not the kernel's tiling) and answers every query of the
``capsule_triangles`` golden fixture plus 200,000 seeded triangles; each
answer must equal the reference's (fixture) and the oracle's bit for bit.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import pyoracle
from golden_util import GOLDEN

HERE = os.path.dirname(os.path.abspath(__file__))
D = C.POINTER(C.c_double)
U8 = C.POINTER(C.c_uint8)


@pytest.fixture(scope='module')
def emu(tmp_path_factory):
    cxx = shutil.which('g++')
    if cxx is None:
        pytest.skip('no host C++ compiler')
    out = str(tmp_path_factory.mktemp('emu') / 'libcapsule_host.so')
    subprocess.run([cxx, '-O2', '-std=c++17', '-fPIC', '-shared', '-ffp-contract=off', '-o', out,
                    os.path.join(HERE, 'emulation', 'capsule_host.cpp')], check=True)
    lib = C.CDLL(out)
    lib.emu_capsule_triangles.argtypes = [D, D, C.c_double, D, C.c_int64, U8, D, D, D]
    lib.emu_capsule_triangles.restype = None
    return lib


def _run(lib, p0, p1, r, verts):
    verts = np.ascontiguousarray(verts, 'd').reshape(-1, 3, 3)
    n = len(verts)
    hit = np.zeros(n, np.uint8)
    pts, nrm, dep = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
    p = lambda a: a.ctypes.data_as(D)
    a, b = np.ascontiguousarray(p0, 'd'), np.ascontiguousarray(p1, 'd')
    lib.emu_capsule_triangles(p(a), p(b), float(r), p(verts), n, hit.ctypes.data_as(U8), p(pts), p(nrm), p(dep))
    return hit.astype(bool), pts, nrm, dep


def test_reference_answers(emu):
    fix = np.load(GOLDEN + '/capsule_triangles.npz')
    off = fix['tri_off']
    for q, c in enumerate(fix['caps']):
        s, e = int(off[q]), int(off[q + 1])
        got = _run(emu, c[:3], c[3:6], c[6], fix['verts'][s:e])
        for g, key in zip(got, ('hit', 'points', 'normals', 'depths')):
            want = fix[key][s:e].astype(bool) if key == 'hit' else fix[key][s:e]
            assert np.array_equal(g, want), (q, key)


def test_seeded_triangles_equal_the_oracle(emu):
    rng = np.random.default_rng(17)
    for k in range(50):
        axis = rng.normal(size=3)
        axis /= np.linalg.norm(axis)
        c = rng.normal(size=3)
        half = rng.uniform(0.0, 0.9)
        p0, p1, r = c - axis * half, c + axis * half, rng.uniform(0.1, 0.9)
        verts = c + rng.normal(scale=rng.uniform(0.5, 2.0), size=(4000, 3, 3))
        verts[::50, 1] = verts[::50, 0]                  # degenerate: repeated vertex
        got = _run(emu, p0, p1, r, verts)
        want = pyoracle.capsule_triangles(p0, p1, r, verts)
        for g, w, key in zip(got, want, ('hit', 'points', 'normals', 'depths')):
            assert np.array_equal(g, w), (k, key)
