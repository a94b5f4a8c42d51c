"""OMI glTF physics documents: read, write, and build worlds from them.

``load_document`` / ``export_extensions`` read and write the
``OMI_physics_shape`` / ``OMI_physics_body`` / ``OMI_physics_gravity`` /
``OMI_physics_joint`` blocks of a glTF JSON dict with the same defaults and
the same output as the reference's ``omi_gltf`` (``src/omi_physics/
omi_gltf.py:45-334``), so a document loads here exactly as it loads there.

``build_world`` turns a document into a world ready to step (the reference
stops at the document): every node with a physics body becomes a body at the
node's translation and rotation, in node order; materials and collision
filters keep their document indices; the document's gravity becomes the
world's; a gravity node becomes a gravity volume bounded by the node's own
sensor shape (a sphere or box) when it has one, else acting everywhere.
``Server.submit_document`` serves documents this way.
"""
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from . import model

SUPPORTED = ('OMI_physics_shape', 'OMI_physics_body', 'OMI_physics_gravity', 'OMI_physics_joint')


@dataclass
class NodeBody:
    """The physics attached to one glTF node; any part may be absent."""
    motion: Optional[model.Motion] = None
    collider: Optional[model.Collider] = None
    trigger: Optional[model.Trigger] = None
    gravity: Optional[model.Gravity] = None
    joint: Optional[model.JointAttach] = None


@dataclass
class PhysicsDocument:
    """Document-level tables plus the physics of each node, by node index."""
    shapes: List[model.Shape] = field(default_factory=list)
    materials: List[model.Material] = field(default_factory=list)
    filters: List[model.CollisionFilter] = field(default_factory=list)
    joints: List[model.Joint] = field(default_factory=list)
    global_gravity: Optional[model.Gravity] = None
    node_bodies: Dict[int, NodeBody] = field(default_factory=dict)


# -- reading -----------------------------------------------------------------
def _shape(entry: dict) -> model.Shape:
    kind = entry['type']
    p = entry.get(kind, {})
    if kind == 'box':
        return model.Shape.box(p.get('size', [1, 1, 1]))
    if kind == 'sphere':
        return model.Shape.sphere(p.get('radius', 0.5))
    if kind == 'capsule':
        return model.Shape.capsule(p.get('height', 1.0), p.get('radius', 0.5))
    if kind == 'cylinder':
        return model.Shape(type='cylinder', height=p.get('height', 2.0),
                           radiusBottom=p.get('radiusBottom', 0.5), radiusTop=p.get('radiusTop', 0.5))
    if kind in ('convex', 'trimesh'):
        return model.Shape(type=kind, mesh=p.get('mesh', -1))
    raise ValueError('unknown OMI shape type %r' % kind)


def _gravity(d: dict) -> model.Gravity:
    return model.Gravity(type=d.get('type', model.DIRECTIONAL), gravity=d.get('gravity', 9.81),
                         direction=tuple(d.get('direction', (0, -1, 0))), priority=d.get('priority', 0),
                         replace=d.get('replace', False), stop=d.get('stop', False),
                         center=tuple(d.get('center', (0, 0, 0))))


def _motion(d: dict) -> model.Motion:
    return model.Motion(type=d['type'], mass=d.get('mass', 1.0),
                        centerOfMass=tuple(d.get('centerOfMass', (0, 0, 0))),
                        inertiaDiagonal=tuple(d.get('inertiaDiagonal', (0, 0, 0))),
                        inertiaOrientation=tuple(d.get('inertiaOrientation', (0, 0, 0, 1))),
                        linearVelocity=tuple(d.get('linearVelocity', (0, 0, 0))),
                        angularVelocity=tuple(d.get('angularVelocity', (0, 0, 0))),
                        gravityFactor=d.get('gravityFactor', 1.0))


def _joint(d: dict) -> model.Joint:
    limits = [model.JointLimit(linearAxes=tuple(x.get('linearAxes', [])),
                               angularAxes=tuple(x.get('angularAxes', [])),
                               min=x.get('min', -np.inf), max=x.get('max', np.inf),
                               stiffness=x.get('stiffness', np.inf), damping=x.get('damping', 0.0))
              for x in d.get('limits', [])]
    drives = [model.JointDrive(type=x.get('type', 'linear'), mode=x.get('mode', 'force'),
                               axis=x.get('axis', 0), maxForce=x.get('maxForce', np.inf),
                               positionTarget=x.get('positionTarget'), velocityTarget=x.get('velocityTarget'),
                               stiffness=x.get('stiffness', 0.0), damping=x.get('damping', 0.0))
              for x in d.get('drives', [])]
    return model.Joint(limits=limits, drives=drives)


def load_document(gltf: dict) -> PhysicsDocument:
    """Every OMI physics block of a glTF JSON dict (omi_gltf.py:220-263)."""
    doc = PhysicsDocument()
    top = gltf.get('extensions', {}) or {}
    doc.shapes = [_shape(e) for e in top.get('OMI_physics_shape', {}).get('shapes', [])]
    body = top.get('OMI_physics_body', {})
    doc.materials = [model.Material(staticFriction=m.get('staticFriction', 0.6),
                                    dynamicFriction=m.get('dynamicFriction', 0.6),
                                    restitution=m.get('restitution', 0.0),
                                    frictionCombine=m.get('frictionCombine', model.AVERAGE),
                                    restitutionCombine=m.get('restitutionCombine', model.AVERAGE))
                     for m in body.get('physicsMaterials', [])]
    doc.filters = [model.CollisionFilter(
        collisionSystems=tuple(f.get('collisionSystems', [])),
        collideWithSystems=tuple(f['collideWithSystems']) if 'collideWithSystems' in f else None,
        notCollideWithSystems=tuple(f.get('notCollideWithSystems', [])))
        for f in body.get('collisionFilters', [])]
    doc.joints = [_joint(j) for j in top.get('OMI_physics_joint', {}).get('physicsJoints', [])]
    if top.get('OMI_physics_gravity'):
        doc.global_gravity = _gravity(top['OMI_physics_gravity'])
    for idx, node in enumerate(gltf.get('nodes', [])):
        ext = node.get('extensions', {}) or {}
        nb, found = NodeBody(), False
        b = ext.get('OMI_physics_body')
        if b:
            found = True
            if 'motion' in b:
                nb.motion = _motion(b['motion'])
            if 'collider' in b:
                c = b['collider']
                nb.collider = model.Collider(shape=c.get('shape', -1), physicsMaterial=c.get('physicsMaterial', -1),
                                             collisionFilter=c.get('collisionFilter', -1))
            if 'trigger' in b:
                nb.trigger = model.Trigger(shape=b['trigger'].get('shape', -1))
            if 'joint' in b:
                j = b['joint']
                nb.joint = model.JointAttach(joint=j.get('joint', -1), connectedNode=j.get('connectedNode', -1),
                                             enableCollision=j.get('enableCollision', False))
        if ext.get('OMI_physics_gravity'):
            found = True
            nb.gravity = _gravity(ext['OMI_physics_gravity'])
        if found:
            doc.node_bodies[idx] = nb
    return doc


# -- writing -----------------------------------------------------------------
def _shape_out(s: model.Shape) -> dict:
    if s.type == 'box':
        return {'type': 'box', 'box': {'size': list(s.size)}}
    if s.type == 'sphere':
        return {'type': 'sphere', 'sphere': {'radius': s.radius}}
    if s.type == 'capsule':
        return {'type': 'capsule', 'capsule': {'height': s.height, 'radius': s.radiusBottom}}
    if s.type == 'cylinder':
        return {'type': 'cylinder', 'cylinder': {'height': s.height, 'radiusBottom': s.radiusBottom,
                                                 'radiusTop': s.radiusTop}}
    return {'type': s.type, s.type: {'mesh': s.mesh}}


def _joint_out(j: model.Joint) -> dict:
    out: Dict[str, list] = {}
    if j.limits:
        lims = []
        for x in j.limits:
            e = {'linearAxes': list(x.linearAxes), 'angularAxes': list(x.angularAxes)}
            if np.isfinite(x.min):
                e['min'] = x.min
            if np.isfinite(x.max):
                e['max'] = x.max
            lims.append(e)
        out['limits'] = lims
    if j.drives:
        drs = []
        for x in j.drives:
            e = {'type': x.type, 'mode': x.mode, 'axis': x.axis}
            if x.positionTarget is not None:
                e['positionTarget'] = x.positionTarget
            if x.velocityTarget is not None:
                e['velocityTarget'] = x.velocityTarget
            if np.isfinite(x.maxForce):
                e['maxForce'] = x.maxForce
            drs.append(e)
        out['drives'] = drs
    return out


def export_extensions(doc: PhysicsDocument) -> Tuple[dict, dict]:
    """``(top-level extensions, {node index: node extensions})`` reproducing the
    OMI blocks (omi_gltf.py:266-300)."""
    top: Dict[str, dict] = {}
    if doc.shapes:
        top['OMI_physics_shape'] = {'shapes': [_shape_out(s) for s in doc.shapes]}
    body: Dict[str, list] = {}
    if doc.materials:
        body['physicsMaterials'] = [{'staticFriction': m.staticFriction, 'dynamicFriction': m.dynamicFriction,
                                     'restitution': m.restitution, 'frictionCombine': m.frictionCombine,
                                     'restitutionCombine': m.restitutionCombine} for m in doc.materials]
    if doc.filters:
        fl = []
        for f in doc.filters:
            e = {'collisionSystems': list(f.collisionSystems),
                 'notCollideWithSystems': list(f.notCollideWithSystems)}
            if f.collideWithSystems is not None:
                e['collideWithSystems'] = list(f.collideWithSystems)
            fl.append(e)
        body['collisionFilters'] = fl
    if body:
        top['OMI_physics_body'] = body
    if doc.joints:
        top['OMI_physics_joint'] = {'physicsJoints': [_joint_out(j) for j in doc.joints]}
    if doc.global_gravity is not None:
        g = doc.global_gravity
        top['OMI_physics_gravity'] = {'gravity': g.gravity, 'direction': list(g.direction)}
    nodes: Dict[int, dict] = {}
    for idx, nb in doc.node_bodies.items():
        ext: Dict[str, dict] = {}
        b: Dict[str, dict] = {}
        if nb.motion is not None:
            m = nb.motion
            b['motion'] = {'type': m.type, 'mass': m.mass, 'centerOfMass': list(m.centerOfMass),
                           'inertiaDiagonal': list(m.inertiaDiagonal),
                           'inertiaOrientation': list(m.inertiaOrientation),
                           'linearVelocity': list(m.linearVelocity), 'angularVelocity': list(m.angularVelocity),
                           'gravityFactor': m.gravityFactor}
        if nb.collider is not None:
            c = {'shape': nb.collider.shape}
            if nb.collider.physicsMaterial >= 0:
                c['physicsMaterial'] = nb.collider.physicsMaterial
            if nb.collider.collisionFilter >= 0:
                c['collisionFilter'] = nb.collider.collisionFilter
            b['collider'] = c
        if nb.trigger is not None:
            b['trigger'] = {'shape': nb.trigger.shape}
        if nb.joint is not None:
            b['joint'] = {'joint': nb.joint.joint, 'connectedNode': nb.joint.connectedNode,
                          'enableCollision': nb.joint.enableCollision}
        if b:
            ext['OMI_physics_body'] = b
        if nb.gravity is not None:
            g = nb.gravity
            v = {'type': g.type, 'gravity': g.gravity, 'priority': g.priority, 'replace': g.replace, 'stop': g.stop}
            if g.type == model.POINT:
                v['center'] = list(g.center)
            else:
                v['direction'] = list(g.direction)
            ext['OMI_physics_gravity'] = v
        nodes[idx] = ext
    return top, nodes


# -- worlds ------------------------------------------------------------------
def build_world(gltf: dict, api=None, backend=None, fixed_dt: float = 1.0 / 60.0,
                mesh_points: Optional[Callable[[int], np.ndarray]] = None):
    """A world holding the document's bodies, ready to step.

    ``api`` is a namespace with ``PhysicsWorld``, ``model`` and ``gravity``
    (this package by default, or the reference's modules, which build the
    identical world). Nodes become bodies in node order at their
    ``translation`` / ``rotation`` (xyzw); a node with a collider or sensor
    but no motion is static. ``mesh_points(mesh)`` supplies a convex shape's
    local points (glTF mesh data is not read here); without it a convex shape
    raises ``ValueError``. Joint attachments stay in the document.
    """
    from .scenes import default_api
    api = api or default_api()
    m, G = api.model, api.gravity
    doc = load_document(gltf)
    kw = {'fixed_dt': fixed_dt}
    if backend is not None:
        kw['backend'] = backend
    if doc.global_gravity is not None:
        g = doc.global_gravity
        kw['gravity'] = m.Gravity(gravity=g.gravity, direction=tuple(g.direction))
    w = api.PhysicsWorld(**kw)
    for s in doc.shapes:
        if s.type == 'convex':
            if mesh_points is None:
                raise ValueError('convex shape on mesh %d needs mesh_points' % s.mesh)
            s = m.Shape.convex(np.asarray(mesh_points(s.mesh), dtype='d'))
        elif s.type == 'cylinder':
            s = m.Shape(type='cylinder', height=s.height, radiusBottom=s.radiusBottom, radiusTop=s.radiusTop)
        elif s.type == 'capsule':
            s = m.Shape.capsule(s.height, s.radiusBottom)
        elif s.type == 'box':
            s = m.Shape.box(tuple(s.size))
        elif s.type == 'sphere':
            s = m.Shape.sphere(s.radius)
        else:
            s = m.Shape(type=s.type, mesh=s.mesh)
        w.add_shape(s)
    for mat in doc.materials:
        w.add_material(m.Material(staticFriction=mat.staticFriction, dynamicFriction=mat.dynamicFriction,
                                  restitution=mat.restitution, frictionCombine=mat.frictionCombine,
                                  restitutionCombine=mat.restitutionCombine))
    for f in doc.filters:
        w.add_filter(m.CollisionFilter(collisionSystems=f.collisionSystems,
                                       collideWithSystems=f.collideWithSystems,
                                       notCollideWithSystems=f.notCollideWithSystems))
    nodes = gltf.get('nodes', [])
    for idx in sorted(doc.node_bodies):
        nb = doc.node_bodies[idx]
        node = nodes[idx]
        pos = tuple(float(x) for x in node.get('translation', (0.0, 0.0, 0.0)))
        rot = tuple(float(x) for x in node.get('rotation', (0.0, 0.0, 0.0, 1.0)))
        if nb.motion is not None or nb.collider is not None or nb.trigger is not None:
            mo = nb.motion
            motion = (m.Motion(type=mo.type, mass=mo.mass, linearVelocity=tuple(mo.linearVelocity),
                               angularVelocity=tuple(mo.angularVelocity), gravityFactor=mo.gravityFactor)
                      if mo is not None else m.Motion(type=m.STATIC))
            col = (m.Collider(shape=nb.collider.shape, physicsMaterial=nb.collider.physicsMaterial,
                              collisionFilter=nb.collider.collisionFilter) if nb.collider is not None else None)
            trg = m.Trigger(shape=nb.trigger.shape) if nb.trigger is not None else None
            w.add_body(motion, col, trigger=trg, position=pos, orientation=rot)
        if nb.gravity is not None:
            gv = nb.gravity
            field_ = m.Gravity(type=gv.type, gravity=gv.gravity, direction=tuple(gv.direction),
                               priority=gv.priority, replace=gv.replace, stop=gv.stop, center=tuple(gv.center))
            region = None
            if nb.trigger is not None and 0 <= nb.trigger.shape < len(doc.shapes):
                sh = doc.shapes[nb.trigger.shape]
                if sh.type == 'sphere':
                    region = G.SphereRegion(pos, sh.radius)
                elif sh.type == 'box':
                    region = G.BoxRegion(pos, tuple(0.5 * np.asarray(sh.size, dtype='d')))
            w.add_gravity_volume(G.GravityVolume(field_, region))
    return w
