"""Malformed scenes are refused on the host, before any device work.

``omi_validate_scene`` runs the same checks ``omi_load`` runs before it
releases the previous arena (no device or context needed): every index a
kernel would follow is range-checked, so a scene that would make a kernel
read out of bounds is refused with OMI_E_ARG and a message, and an
unsupported feature with OMI_E_UNSUPPORTED. Each case below plants one fault
in the packed tables of an otherwise valid two-world scene (a debris world
and a jointed chain).
"""
import numpy as np
import pytest

from omi_physics_b200 import _lib, scenes
from omi_physics_b200.arena import pack_worlds


@pytest.fixture(scope='module', autouse=True)
def library():
    from omi_physics_b200 import build
    build.build()


def _packed():
    a, ma = scenes.debris(n=40, seed=3)
    b, mb = scenes.joint_chain(links=6, loose=8, seed=2)
    return pack_worlds([a, b], [ma['dt'], mb['dt']])


def test_valid_scene_passes():
    P = _packed()                  # keeps the arrays the scene points at alive
    _lib.validate_scene(P.scene)


def _refused(mutate, code=_lib.OMI_E_ARG, words=()):
    P = _packed()
    mutate(P)
    with pytest.raises(_lib.OmiError) as e:
        _lib.validate_scene(P.scene)
    assert e.value.code == code
    for w in words:
        assert w in str(e.value)


def test_shape_index_out_of_range():
    def m(P):
        P.arrays['shape'][5] = P.scene.n_shapes
    _refused(m, words=('shape index',))


def test_shape_index_below_minus_one():
    def m(P):
        P.arrays['shape'][5] = -7
    _refused(m, words=('shape index',))


def test_material_index_out_of_range():
    def m(P):
        P.arrays['material'][3] = P.scene.n_materials + 2
    _refused(m, words=('material',))


def test_motion_type_out_of_range():
    def m(P):
        P.arrays['motion_type'][4] = 3
    _refused(m, words=('motion type',))


def test_filter_row_out_of_range():
    def m(P):
        P.arrays['filter_row'][2] = 9
    _refused(m, words=('filter row',))


def test_world_offsets_inconsistent():
    def m(P):
        P.arrays['w_body_off'][-1] += 1
    _refused(m, words=('offsets',))


def test_joint_body_out_of_range():
    def m(P):
        P.arrays['j_a'][0] = P.scene.n_bodies + 5
    _refused(m, words=('joint body',))


def test_joint_body_below_minus_one():
    def m(P):
        P.arrays['j_b'][1] = -3
    _refused(m, words=('joint body',))


def test_joint_body_in_another_world():
    # the chain's joints belong to world 1; body 2 is in world 0
    def m(P):
        P.arrays['j_a'][0] = 2
    _refused(m, words=("joint's world",))


def test_convex_point_range_out_of_bounds():
    w, meta = scenes.convex_pile(n=24, seed=1)
    P = pack_worlds([w], [meta['dt']])
    hull = int(np.flatnonzero(P.arrays['shape_pt_cnt'] > 0)[0])
    P.arrays['shape_pt_off'][hull] = P.scene.n_points
    with pytest.raises(_lib.OmiError) as e:
        _lib.validate_scene(P.scene)
    assert e.value.code == _lib.OMI_E_ARG and 'point range' in str(e.value)


def test_unknown_shape_type_is_unsupported():
    def m(P):
        P.arrays['shape_type'][P.arrays['shape'][3]] = 42
    _refused(m, code=_lib.OMI_E_UNSUPPORTED)


def test_negative_iterations():
    def m(P):
        P.arrays['w_iters'][1] = -1
    _refused(m, words=('iteration',))


def test_filter_matrix_range():
    def m(P):
        P.arrays['w_filter_off'][1] = P.scene.n_filter_bytes
    _refused(m, words=('filter matrix',))
