"""OMI glTF physics documents (no GPU).

``tests/golden/omi_document.json`` holds a document exercising every shape
kind, materials, filters, a joint table, global gravity, static / kinematic /
dynamic bodies, sensors and gravity-volume nodes, together with the
reference's own export of it (``omi_gltf.load_document`` +
``export_extensions``) and the columns of the world built from it with the
reference's classes. Reading and re-writing here must reproduce the
reference's export exactly, re-export must be stable, and the world built
here must have the reference world's columns.
"""
import copy
import json

import numpy as np
import pytest

from golden_util import GOLDEN
from omi_physics_b200 import gltf, model

FIX = json.load(open(GOLDEN + '/omi_document.json'))


def test_export_equals_the_references():
    doc = gltf.load_document(FIX['gltf'])
    top, nodes = gltf.export_extensions(doc)
    assert top == FIX['export_top']
    assert {str(k): v for k, v in nodes.items()} == FIX['export_nodes']


def test_reexport_is_stable():
    doc = gltf.load_document(FIX['gltf'])
    top, nodes = gltf.export_extensions(doc)
    again = copy.deepcopy(FIX['gltf'])
    again['extensions'] = top
    for idx, ext in nodes.items():
        again['nodes'][idx]['extensions'] = ext
    assert gltf.export_extensions(gltf.load_document(again)) == (top, nodes)


def test_reads_fields_and_defaults():
    doc = gltf.load_document(FIX['gltf'])
    kinds = [s.type for s in doc.shapes]
    assert {'box', 'sphere', 'capsule', 'cylinder', 'trimesh'} <= set(kinds)
    assert doc.materials[1].frictionCombine == model.MINIMUM
    assert doc.filters[1].collideWithSystems == ('ground',)
    assert doc.filters[0].collideWithSystems is None
    assert doc.joints[0].drives[0].velocityTarget == 2.0
    assert doc.joints[0].limits[1].min == -np.inf              # omitted -> default
    assert doc.global_gravity.gravity == 9.81
    assert doc.node_bodies[1].gravity.type == 'point'
    assert doc.node_bodies[4].joint.connectedNode == 0
    empty = gltf.load_document({'nodes': [{'name': 'plain'}]})
    assert empty.shapes == [] and empty.node_bodies == {}
    with pytest.raises(ValueError):
        gltf.load_document({'extensions': {'OMI_physics_shape': {'shapes': [{'type': 'cone'}]}}})


def test_world_built_here_equals_the_reference_world():
    plain = dict(FIX['gltf'], nodes=[nd for nd in FIX['gltf']['nodes'] if nd['name'] != 'mesh'])
    w = gltf.build_world(plain, fixed_dt=1.0 / 120.0)
    n = w.body_count
    for name, want in FIX['world_init'].items():
        got = np.asarray(getattr(w, '_' + name)[:n])
        assert np.array_equal(got, np.asarray(want, dtype=got.dtype)), name
    assert len(w.gravity_volumes) == FIX['volumes'] == 3
    regions = sorted(type(v.region).__name__ for v in w.gravity_volumes)
    assert regions == ['BoxRegion', 'InfiniteRegion', 'SphereRegion']


def test_convex_shapes_need_mesh_points():
    doc = {'extensions': {'OMI_physics_shape': {'shapes': [{'type': 'convex', 'convex': {'mesh': 7}}]}},
           'nodes': [{'translation': [0, 2, 0], 'extensions': {'OMI_physics_body': {
               'motion': {'type': 'dynamic'}, 'collider': {'shape': 0}}}}]}
    with pytest.raises(ValueError):
        gltf.build_world(doc)
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], 'd')
    w = gltf.build_world(doc, mesh_points=lambda mesh: pts if mesh == 7 else None)
    assert w.body_count == 1 and w.shapes[0].type == 'convex'
    assert np.array_equal(w.shapes[0].points, pts)
