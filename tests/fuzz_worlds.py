"""Seeded random worlds for the fuzz tests: every shape kind, motion type,
friction and restitution combine mode, a pair-friction override, collision
filters, damping / drag / gravity factors, sensors on every motion type, a
resting stack that falls asleep, and gravity volumes of every kind. ``api``
is a namespace with ``PhysicsWorld``, ``model`` and ``gravity`` of either the
reference or this package, which build identical worlds."""
import numpy as np


def _quat(rng):
    q = rng.normal(size=4)
    return tuple(float(x) for x in q / np.linalg.norm(q))


def random_world(api, seed, n=40):
    m, G = api.model, api.gravity
    rng = np.random.default_rng(seed)
    w = api.PhysicsWorld(fixed_dt=1.0 / 120.0, default_linear_damping=float(rng.choice([0.0, 0.02])))
    modes = (m.AVERAGE, m.MINIMUM, m.MAXIMUM, m.MULTIPLY)
    mats = [w.add_material(m.Material(staticFriction=float(rng.uniform(0.1, 1.0)),
                                      dynamicFriction=float(rng.uniform(0.05, 0.9)),
                                      restitution=float(rng.choice([0.0, 0.2, 0.7])),
                                      frictionCombine=modes[k % 4], restitutionCombine=modes[(k + 1) % 4]))
            for k in range(5)]
    w.set_pair_friction(mats[0], mats[1], 0.8, 0.7)
    filters = [-1,
               w.add_filter(m.CollisionFilter(collisionSystems=('a',), notCollideWithSystems=('b',))),
               w.add_filter(m.CollisionFilter(collisionSystems=('b',))),
               w.add_filter(m.CollisionFilter(collisionSystems=('c',), collideWithSystems=('c', 'a')))]
    ground = w.add_shape(m.Shape.box((14.0, 1.0, 14.0)))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=ground, physicsMaterial=mats[0]),
               position=(0.0, -0.5, 0.0))

    def shape():
        k = rng.integers(0, 5)
        if k == 0:
            return w.add_shape(m.Shape.box(tuple(float(x) for x in rng.uniform(0.3, 1.4, 3))))
        if k == 1:
            return w.add_shape(m.Shape.sphere(float(rng.uniform(0.2, 0.7))))
        if k == 2:
            return w.add_shape(m.Shape.capsule(float(rng.uniform(0.3, 1.2)), float(rng.uniform(0.15, 0.4))))
        if k == 3:
            return w.add_shape(m.Shape.cylinder(float(rng.uniform(0.4, 1.2)), float(rng.uniform(0.2, 0.5))))
        pts = rng.normal(size=(int(rng.integers(8, 20)), 3))
        pts *= rng.uniform(0.3, 0.8, 3) / np.linalg.norm(pts, axis=1, keepdims=True)
        return w.add_shape(m.Shape.convex(pts))

    for i in range(n):
        u = rng.random()
        kind = m.STATIC if u < 0.08 else (m.KINEMATIC if u < 0.16 else m.DYNAMIC)
        pos = tuple(float(x) for x in rng.uniform((-2.5, 0.3, -2.5), (2.5, 3.0, 2.5)))
        motion = m.Motion(type=kind, mass=float(rng.uniform(0.5, 4.0)),
                          linearVelocity=tuple(float(x) for x in rng.normal(0.0, 0.6, 3)) if kind != m.STATIC
                          else (0.0, 0.0, 0.0),
                          angularVelocity=tuple(float(x) for x in rng.normal(0.0, 0.4, 3)) if kind != m.STATIC
                          else (0.0, 0.0, 0.0),
                          linearDamping=float(rng.choice([0.0, 0.1])), angularDamping=float(rng.choice([0.0, 0.2])),
                          quadraticDrag=float(rng.choice([0.0, 0.03])), gravityFactor=float(rng.choice([1.0, 0.5, 1.5])))
        collider = None if rng.random() < 0.05 else m.Collider(shape=shape(), physicsMaterial=mats[i % 5],
                                                              collisionFilter=filters[i % 4])
        trigger = m.Trigger(shape=shape()) if rng.random() < 0.12 else None
        if collider is None and trigger is None and kind == m.STATIC:
            continue
        w.add_body(motion, collider, trigger=trigger, position=pos, orientation=_quat(rng))
    unit = w.add_shape(m.Shape.box((1.0, 1.0, 1.0)))
    for k in range(4):                  # a resting stack that falls asleep unless something hits it
        w.add_body(m.Motion(type=m.DYNAMIC), m.Collider(shape=unit, physicsMaterial=mats[0]),
                   position=(5.5, 0.5 + k, 5.5))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(type='point', gravity=5.0, center=(2.0, 2.0, 0.0), priority=1),
                                         G.SphereRegion((2.0, 2.0, 0.0), 2.5)))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(gravity=3.0, direction=(0.3, 1.0, 0.0), priority=2,
                                                   replace=True), G.BoxRegion((-2.5, 2.0, 2.5), (1.5, 2.0, 1.5))))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(priority=3, stop=True), G.BoxRegion((2.5, 1.5, -2.5), (1.0, 1.5, 1.0))))
    w.add_gravity_volume(G.GravityVolume(m.Gravity(gravity=0.4, direction=(0.0, 0.0, 1.0))))
    w._collision.solver.velocity_iterations = int(rng.integers(4, 11))
    return w


def switch_worlds(api):
    """Small debris worlds, one per world-level switch the step branches on:
    sleeping disabled, warm start off, default damping, no velocity
    iterations, a tilted weaker world gravity, and bodies with no collider at
    all (the world then has no collision stage). ``[(name, world), ...]``."""
    from omi_physics_b200 import scenes
    m = api.model
    out = []
    for k, name in enumerate(('no_sleep', 'no_warm_start', 'default_damping', 'no_iterations', 'tilted_gravity')):
        w, _ = scenes.debris(api, n=60, seed=40 + k, extent=2.5, height=3.0, ground=12.0)
        if name == 'no_sleep':
            w.sleep_enabled = False
        elif name == 'no_warm_start':
            w._collision.solver.warm_start = False
        elif name == 'default_damping':
            w.default_linear_damping = 0.05
            w.default_angular_damping = 0.1
        elif name == 'no_iterations':
            w._collision.solver.velocity_iterations = 0
        else:
            w.gravity = m.Gravity(gravity=5.0, direction=(0.3, -1.0, 0.2))
        out.append((name, w))
    w = api.PhysicsWorld(fixed_dt=1.0 / 120.0, default_linear_damping=0.02)
    rng = np.random.default_rng(47)
    for i in range(20):
        w.add_body(m.Motion(type=m.DYNAMIC if i % 4 else m.KINEMATIC, mass=1.0,
                            linearVelocity=tuple(float(v) for v in rng.normal(0.0, 1.0, 3)),
                            angularVelocity=tuple(float(v) for v in rng.normal(0.0, 1.0, 3)),
                            quadraticDrag=0.05 * (i % 3)),
                   None, position=tuple(float(v) for v in rng.uniform(-3.0, 3.0, 3)))
    out.append(('no_colliders', w))
    return out


def joint_world(api, seed):
    """Boxes and spheres tied by random joints: point joints between two bodies
    and to the world, distance joints, angular motors (``api`` also needs
    ``joints``)."""
    m, J = api.model, api.joints
    rng = np.random.default_rng(seed)
    w = api.PhysicsWorld(fixed_dt=1.0 / 240.0)
    mat = w.add_material(m.Material(staticFriction=0.5, dynamicFriction=0.4))
    w.add_body(m.Motion(type=m.STATIC), m.Collider(shape=w.add_shape(m.Shape.box((20.0, 1.0, 20.0))),
                                                   physicsMaterial=mat), position=(0.0, -0.5, 0.0))
    first = w.body_count
    n = 16
    pos = rng.uniform((-3.0, 1.0, -3.0), (3.0, 5.0, 3.0), size=(n, 3))
    for i in range(n):
        shape = (m.Shape.box(tuple(float(v) for v in rng.uniform(0.3, 0.8, 3))) if i % 2 else
                 m.Shape.sphere(float(rng.uniform(0.2, 0.4))))
        w.add_body(m.Motion(type=m.DYNAMIC, mass=float(rng.uniform(0.5, 3.0))),
                   m.Collider(shape=w.add_shape(shape), physicsMaterial=mat),
                   position=tuple(float(v) for v in pos[i]), orientation=_quat(rng))
    for k in range(10):
        a, b = (int(x) + first for x in rng.choice(n, size=2, replace=False))
        if k < 6:
            mid = tuple(float(v) for v in 0.5 * (pos[a - first] + pos[b - first]))
            w.add_joint_constraint(J.PointConstraint(a, b, mid))
        else:
            w.add_joint_constraint(J.DistanceConstraint(a, b, tuple(float(v) for v in rng.uniform(-0.2, 0.2, 3)),
                                                        tuple(float(v) for v in rng.uniform(-0.2, 0.2, 3))))
    for k in range(3):
        i = first + k
        anchor = tuple(float(v) for v in pos[k] + (0.0, 0.6, 0.0))
        w.add_joint_constraint(J.PointConstraint(-1, i, anchor) if k % 2 == 0 else J.PointConstraint(i, -1, anchor))
    for k in range(3):
        w.add_joint_constraint(J.AngularMotor(first + 5 + k, tuple(float(v) for v in rng.normal(size=3)), 1.5,
                                              max_force=float(rng.choice([5.0, 50.0]))))
    w.joint_iterations = int(rng.integers(6, 13))
    return w
