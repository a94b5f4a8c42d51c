"""The bounds-checked debug library on the GPU (``OMI_B200_CHECKED=1``).

A child process loads ``_omi_b200_checked.so`` and (1) steps worlds that
reach every instrumented kernel - boxes and spheres (pair bodies, filter
rows, solver prep, the per-world sweep, islands), hulls (shape and point
ranges of the GJK/EPA proxies), distance joints and motors, and the same
debris as a wide world swept by the many-block and the one-block sweeps -
each against the oracle every step, bit for bit, with no check failing; (2)
makes one check fail on purpose through the build's test hook (a candidate
pair whose first body is checked as if past the arena): the step raises
``BoundsError`` naming that check and index, nothing faults, and with the
hook off the same context steps on cleanly.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import os, sys
import numpy as np
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
import pyoracle
from omi_physics_b200 import WorldBatch, scenes, _lib
assert _lib.LIB_PATH == _lib.LIB_PATH_CHECKED and _lib.load_library().omi_bounds_checked() == 1

def run(name, builder, steps, launch=None):
    w, meta = builder()
    dt = meta['dt']
    o = pyoracle.OracleWorld.from_world(w)
    b = WorldBatch([w], dts=[dt])
    if launch:
        b.ctx.set_tuning(**launch)
    for s in range(steps):
        b.step(1)                       # raises BoundsError if any check failed
        o.step(dt)
    b.sync_to_host()
    st = o.state()
    assert np.array_equal(b.pairs(0), o.pairs()), name
    for col in ('position', 'orientation', 'linear_velocity', 'angular_velocity', 'sleep_timer'):
        assert np.array_equal(getattr(w, col), st[col]), (name, col)
    assert np.array_equal(w.awake, st['awake']), name
    print('clean', name, steps)

debris = lambda: scenes.debris(n=512, seed=1, extent=8.0, height=12.0, ground=30.0)
run('pyramid', lambda: scenes.pyramid(), 60)
run('debris512', debris, 90)
run('convex160', lambda: scenes.convex_pile(n=160, seed=2, arena=10.0, height=8.0), 60)
run('rods', lambda: scenes.rods(), 60)
os.environ['OMI_WIDE_THRESHOLD'] = '0'            # every colliding world wide
run('debris512 wide, many-block sweep', debris, 60, dict(wide_cluster=0, wide_sweep_blocks=8))
run('debris512 wide, one-block sweep', debris, 60, dict(wide_cluster=0, wide_sweep_blocks=1))
del os.environ['OMI_WIDE_THRESHOLD']

w, meta = scenes.pyramid()
b = WorldBatch([w], dts=[meta['dt']])
b.step(1)
b.ctx.call('bounds_probe', 0)
try:
    b.step(1)
    raise AssertionError('the probed check did not fail')
except _lib.BoundsError as e:
    msg = str(e)
    assert 'narrowphase pair body' in msg and '(index %d)' % b.packed.n_bodies in msg, msg
finally:
    b.ctx.call('bounds_probe', -1)
b.step(5)
print('probe ok:', msg)
'''


def test_checked_build_is_clean_on_real_worlds_and_reports_a_failed_check():
    from omi_physics_b200 import build
    build.build(checked=True)                 # a no-op when it is up to date
    env = dict(os.environ, OMI_B200_CHECKED='1', PYTHONPATH=ROOT)
    env.pop('OMI_WIDE_THRESHOLD', None)
    res = subprocess.run([sys.executable, '-c', 'ROOT = %r\n' % ROOT + CHILD], env=env, cwd=ROOT,
                         capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    assert 'probe ok' in res.stdout
