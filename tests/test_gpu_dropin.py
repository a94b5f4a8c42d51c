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
                                         ('rods', 60), ('convex', 60), ('chain', 60)])
def test_reference_world_steps_on_cuda_backend(scene, steps):
    from omi_physics_b200.backend import CudaBackend
    api = _ref_api()
    gpu, meta = scenes.GOLDEN_SCENES[scene](api, CudaBackend())
    cpu, _ = scenes.GOLDEN_SCENES[scene](api)
    _step_twins(gpu, cpu, meta['dt'], steps, scene)


def _step_twins(gpu, cpu, dt, steps, scene, first=0):
    assert gpu.backend.name == 'cuda' and gpu._backend_mode == 'fixed'
    n = cpu.body_count
    gev, cev = [], []
    gpu.add_trigger_listener(lambda *e: gev.append(e))
    cpu.add_trigger_listener(lambda *e: cev.append(e))
    for s in range(first, first + steps):
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


def test_body_added_mid_run_through_the_drop_in():
    """A topology change between steps: both twins get the same new bodies
    after 25 steps (a box dropped onto the pile and a sphere resting on the
    ground), the CUDA backend reloads its arena and carries the warm-start
    cache over as the reference's solver keeps it (indices do not move,
    solver.py:91, 272-278), and the twins keep agreeing for 45 more steps."""
    from omi_physics_b200.backend import CudaBackend
    api = _ref_api()
    m = api.model
    gpu, meta = scenes.GOLDEN_SCENES['debris'](api, CudaBackend())
    cpu, _ = scenes.GOLDEN_SCENES['debris'](api)
    dt = meta['dt']
    _step_twins(gpu, cpu, dt, 25, 'debris before add')
    for w in (gpu, cpu):
        box = w.add_shape(m.Shape.box((0.8, 0.6, 1.1)))
        ball = w.add_shape(m.Shape.sphere(0.4))
        mat = w.add_material(m.Material(staticFriction=0.6, dynamicFriction=0.6))
        w.add_body(m.Motion(type=m.DYNAMIC, mass=400.0), m.Collider(shape=box, physicsMaterial=mat),
                   position=(0.3, 4.0, -0.2))
        w.add_body(m.Motion(type=m.DYNAMIC, mass=250.0), m.Collider(shape=ball, physicsMaterial=mat),
                   position=(2.0, 0.45, 1.5))
    _step_twins(gpu, cpu, dt, 45, 'debris after add', first=25)
