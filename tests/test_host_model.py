"""Host side without a GPU: the package's PhysicsWorld mirror builds the same
columns as the reference (pinned by the golden fixtures' ``init/*``
snapshots, which the reference wrote), arena packing remaps indices per
world, and features outside the device step are rejected loudly."""
import numpy as np
import pytest

from golden_util import SCENES, load
from omi_physics_b200 import scenes
from omi_physics_b200._lib import UnsupportedFeature
from omi_physics_b200.arena import check_supported, pack_worlds
from omi_physics_b200.backend import CudaBackend, select_backend

COLUMNS = ('position', 'orientation', 'linear_velocity', 'angular_velocity', 'inv_inertia',
           'inv_mass', 'mass', 'gravity_factor', 'linear_damping', 'angular_damping',
           'quadratic_drag', 'sleep_timer', 'motion_type', 'collider_shape', 'collider_material',
           'collider_filter', 'trigger_shape', 'awake')


@pytest.mark.parametrize('scene', SCENES)
def test_mirror_world_columns_equal_reference_init(scene):
    g = load(scene)
    w, _ = scenes.GOLDEN_SCENES[scene]()
    n = w.body_count
    assert n == len(g['init/position'])
    for col in COLUMNS:
        mine = np.asarray(getattr(w, '_' + col)[:n])
        ref = g['init/' + col]
        assert np.array_equal(mine, ref.astype(mine.dtype)), col


def test_pack_two_worlds_offsets_and_remaps():
    a, _ = scenes.GOLDEN_SCENES['pyramid']()
    b, _ = scenes.GOLDEN_SCENES['chain']()
    p = pack_worlds([a, b], [1 / 60, 1 / 240])
    s = p.scene
    na, nb = a.body_count, b.body_count
    assert s.n_worlds == 2 and s.n_bodies == na + nb
    off = p.arrays['w_body_off']
    assert list(off) == [0, na, na + nb]
    shape = p.arrays['shape']
    ok = shape[na:] >= 0
    assert np.array_equal(shape[na:][ok] - len(a.shapes), np.asarray(b._collider_shape[:nb])[ok])
    ja = p.arrays['j_a']
    assert s.n_joints == len(b.joint_constraints)
    assert ((ja < 0) | ((ja >= na) & (ja < na + nb))).all()     # chain joints index world b's rows
    assert np.array_equal(p.arrays['w_dt'], [1 / 60, 1 / 240])


def test_unsupported_features_raise():
    from omi_physics_b200 import model
    w, _ = scenes.GOLDEN_SCENES['pyramid']()
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1]], dtype='d')
    mesh = w.add_shape(model.Shape(type='trimesh', points=pts, indices=np.array([[0, 1, 2]], 'i')))
    w.add_body(model.Motion(type=model.DYNAMIC), model.Collider(shape=mesh), position=(0, 5, 0))
    with pytest.raises(UnsupportedFeature):
        check_supported(w)                        # a moving triangle mesh
    with pytest.raises(UnsupportedFeature):
        CudaBackend().attach(w)
    w5, _ = scenes.GOLDEN_SCENES['terrain']()
    check_supported(w5)                           # static meshes are taken
    w2, _ = scenes.GOLDEN_SCENES['pyramid']()
    s = w2.add_shape(model.Shape(type='trimesh', points=pts, indices=np.array([[0, 1, 2]], 'i')))
    w2.add_body(model.Motion(type=model.STATIC), trigger=model.Trigger(shape=s), position=(0, 9, 0))
    with pytest.raises(UnsupportedFeature):
        check_supported(w2)                       # a triangle-mesh sensor
    w3, _ = scenes.GOLDEN_SCENES['pyramid']()
    w3.add_gravity_volume(object())
    with pytest.raises(UnsupportedFeature):
        check_supported(w3)                       # not a gravity volume
    w4, _ = scenes.GOLDEN_SCENES['zones']()
    check_supported(w4)                           # box / sphere / capsule sensors, all four volume kinds


def test_select_backend_has_no_fallback():
    assert isinstance(select_backend('cuda'), CudaBackend)
    with pytest.raises(ValueError):
        select_backend('numpy')


def test_pack_with_empty_and_static_only_worlds():
    api = scenes.default_api()
    m = api.model
    empty = api.PhysicsWorld(fixed_dt=1 / 60)
    statics = api.PhysicsWorld(fixed_dt=1 / 60)
    slab = statics.add_shape(m.Shape.box((4.0, 1.0, 4.0)))
    statics.add_body(m.Motion(type=m.STATIC), m.Collider(shape=slab), position=(0.0, -0.5, 0.0))
    deg, _ = scenes.degenerate()
    p = pack_worlds([empty, statics, deg, empty])
    off = p.arrays['w_body_off']
    assert list(off) == [0, 0, 1, 1 + deg.body_count, 1 + deg.body_count]
    assert p.scene.n_worlds == 4 and p.scene.n_bodies == 1 + deg.body_count
    p0 = pack_worlds([empty])
    assert p0.scene.n_bodies == 0 and list(p0.arrays['w_body_off']) == [0, 0]


def test_reload_after_a_topology_change_keeps_the_warm_start_cache(monkeypatch):
    """Adding a body changes the world's static signature and reloads the
    arena; the warm-start cache of the last step must carry over, as the
    reference's solver keeps it (solver.py:91, 272-278). Host logic only: a
    stand-in batch records the calls."""
    import omi_physics_b200.batch as batch_mod
    made = []

    class FakeBatch:
        def __init__(self, worlds, device=0, dts=None, ctx=None):
            self.ctx, self.dts, self.set = ctx or object(), dts, None
            self.entries = dict(a=np.array([1], np.int32), b=np.array([2], np.int32),
                                point=np.zeros((1, 3)), impulse=np.array([[3.0, 0.5, -0.5]]))
            made.append(self)

        def cache(self, i):
            return self.entries

        def set_cache(self, i, a, b, point, impulse):
            self.set = (a, b, point, impulse)

        def upload_state(self, i):
            pass

        def refresh_params(self):
            pass

    monkeypatch.setattr(batch_mod, 'WorldBatch', FakeBatch)
    w, meta = scenes.pyramid(levels=3)
    be = CudaBackend()
    be.attach(w)
    be._ensure_loaded(w, meta['dt'])
    assert len(made) == 1 and made[0].set is None        # a first load has nothing to carry
    be._ensure_loaded(w, meta['dt'])
    assert len(made) == 1                                # same topology: no reload
    m = scenes.default_api().model
    w.add_body(m.Motion(type=m.DYNAMIC), m.Collider(shape=1), position=(0.0, 9.0, 0.0))
    be._ensure_loaded(w, meta['dt'])
    assert len(made) == 2 and made[1].ctx is made[0].ctx  # reloaded into the same context
    a, b, point, impulse = made[1].set
    assert list(a) == [1] and list(b) == [2] and np.array_equal(impulse, [[3.0, 0.5, -0.5]])
