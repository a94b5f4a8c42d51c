"""The drop-in: ``CudaBackend`` inside the reference's own ``PhysicsWorld``.

The reference (built from its sources into ``oracle/_ref``) takes an object
backend as fixed (world.py:335-338). One reference world steps with the CUDA
backend, a twin with the reference's default CPU path (its Cython
accelerators); pair sets, contact counts, sleep flags and the trigger
events dispatched to listeners (as sets per step) must match exactly,
poses within 1e-6 m over 60 steps and contact normals/depths within 1e-9.
Skipped when the reference has not been built here.
"""
import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

from omi_physics_b200 import scenes

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, 'oracle', '_ref')


def _ref_api():
    if not os.path.isdir(os.path.join(REF, 'omi_physics')):
        pytest.skip('the reference is not built (oracle/build_ref.sh)')
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import omi_physics as ref
    from omi_physics import gravity, joints, model
    return SimpleNamespace(PhysicsWorld=ref.PhysicsWorld, model=model, joints=joints, gravity=gravity)


@pytest.mark.parametrize('scene,steps', [('pyramid', 60), ('debris', 60), ('spheres', 60),
                                         ('capsules', 30), ('zones', 60), ('terrain', 40),
                                         ('conveyor', 40), ('degenerate', 140),
                                         ('rods', 60)])
def test_reference_world_steps_on_cuda_backend(scene, steps):
    from omi_physics_b200.backend import CudaBackend
    api = _ref_api()
    gpu, meta = scenes.GOLDEN_SCENES[scene](api, CudaBackend())
    cpu, _ = scenes.GOLDEN_SCENES[scene](api)
    dt = meta['dt']
    assert gpu.backend.name == 'cuda' and gpu._backend_mode == 'fixed'
    n = cpu.body_count
    gev, cev = [], []
    gpu.add_trigger_listener(lambda *e: gev.append(e))
    cpu.add_trigger_listener(lambda *e: cev.append(e))
    for s in range(steps):
        gev.clear()
        cev.clear()
        gpu.step(dt)
        cpu.step(dt)
        tag = '%s step %d' % (scene, s)
        assert sorted(gev) == sorted(cev), tag + ' trigger events'
        gp = gpu._collision.broadphase.pairs(gpu)
        cp = [tuple(map(int, p)) for p in cpu._collision.broadphase.pairs(cpu)]
        assert gp == cp, tag + ' pairs (set and order)'
        assert np.array_equal(gpu._awake[:n], cpu._awake[:n]), tag + ' sleep flags'
        assert len(gpu.contacts) == len(cpu.contacts), tag + ' contact count'
        if len(cpu.contacts):
            gn = np.array([c.normal for c in gpu.contacts])
            cn = np.array([c.normal for c in cpu.contacts])
            assert np.allclose(gn, cn, rtol=1e-9, atol=1e-12), tag + ' normals'
            gd = np.array([c.depth for c in gpu.contacts])
            cd = np.array([c.depth for c in cpu.contacts])
            assert np.allclose(gd, cd, rtol=1e-9, atol=1e-12), tag + ' depths'
        assert np.max(np.abs(gpu._position[:n] - cpu._position[:n]), initial=0.0) <= 1e-6, tag + ' pos'
        assert np.max(np.abs(gpu._orientation[:n] - cpu._orientation[:n]), initial=0.0) <= 1e-6, tag


def test_reference_empty_world_on_cuda_backend():
    from omi_physics_b200.backend import CudaBackend
    api = _ref_api()
    gpu = api.PhysicsWorld(fixed_dt=1.0 / 60.0, backend=CudaBackend())
    cpu = api.PhysicsWorld(fixed_dt=1.0 / 60.0)
    for _ in range(3):
        gpu.step(1.0 / 60.0)
        cpu.step(1.0 / 60.0)
    assert gpu.body_count == cpu.body_count == 0
    assert len(gpu.contacts) == len(cpu.contacts) == 0
    assert gpu.time == cpu.time
