"""The reference's own known-answer tests for this path, restated against the
oracle with the same inputs, expectations and tolerances: from the
reference's tests/test_physics_integrate.py (closed-form free fall, gravity
factor, constant velocity, static bodies, damping and drag terminal
velocities), tests/test_collide_primitives.py (sphere and box contacts),
tests/test_solver.py (rest, bounce, a resting stack, friction on an incline,
determinism), tests/test_gravity.py (point pull, priority replace, stop,
region bounds), tests/test_triggers.py (enter / stay / exit, no impulse),
tests/test_joints.py (rods, pins, motors and their force limit) and
tests/test_broadphase.py (pairs equal to brute force). Worlds are built with
this package's world mirror, whose columns equal the reference's; the oracle
steps them.
"""
import math

import numpy as np
import pytest

import pyoracle
from omi_physics_b200 import scenes

API = scenes.default_api()
M = API.model


def _run(world, dt, steps):
    o = pyoracle.OracleWorld.from_world(world)
    for _ in range(steps):
        o.step(dt)
    return o.state()


# -- integration (test_physics_integrate.py) ------------------------------------
def test_freefall_matches_symplectic_closed_form():
    g, dt, n = 9.81, 1.0 / 240.0, 240
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=g, direction=(0, -1, 0)))
    i = w.add_body(M.Motion(type=M.DYNAMIC), position=(0, 0, 0))
    st = _run(w, dt, n)
    assert st['position'][i][1] == pytest.approx(-0.5 * g * dt * dt * n * (n + 1), rel=1e-9)


def test_freefall_approaches_analytic_as_dt_shrinks():
    g, dt = 9.81, 1.0 / 2000.0
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=g, direction=(0, -1, 0)))
    i = w.add_body(M.Motion(type=M.DYNAMIC), position=(0, 0, 0))
    st = _run(w, dt, int(1.0 / dt))
    assert st['position'][i][1] == pytest.approx(-0.5 * g, rel=2e-3)


def test_gravity_factor_scales_fall():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=10.0, direction=(0, -1, 0)))
    full = w.add_body(M.Motion(type=M.DYNAMIC, gravityFactor=1.0), position=(0, 0, 0))
    half = w.add_body(M.Motion(type=M.DYNAMIC, gravityFactor=0.5), position=(0, 0, 0))
    st = _run(w, 1.0 / 240.0, 240)
    assert st['position'][half][1] == pytest.approx(0.5 * st['position'][full][1], rel=1e-9)


def test_zero_net_force_keeps_constant_velocity():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=0.0))
    i = w.add_body(M.Motion(type=M.DYNAMIC, linearVelocity=(2.0, 0.0, -3.0)), position=(0, 0, 0))
    st = _run(w, 1.0 / 120.0, 120)
    assert np.allclose(st['linear_velocity'][i], (2.0, 0.0, -3.0))
    assert np.allclose(st['position'][i], (2.0, 0.0, -3.0), atol=1e-9)


def test_static_body_never_moves():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=9.81))
    i = w.add_body(M.Motion(type=M.STATIC), position=(1, 2, 3))
    assert np.allclose(_run(w, 1 / 60, 100)['position'][i], (1, 2, 3))


def test_linear_damping_terminal_velocity():
    g, c = 9.81, 2.0
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=g, direction=(0, -1, 0)))
    i = w.add_body(M.Motion(type=M.DYNAMIC, linearDamping=c), position=(0, 0, 0))
    st = _run(w, 1.0 / 240.0, 4000)
    assert abs(st['linear_velocity'][i][1]) == pytest.approx(g / c, rel=1e-2)


def test_quadratic_drag_terminal_velocity():
    g, k = 9.81, 0.5
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=g, direction=(0, -1, 0)))
    i = w.add_body(M.Motion(type=M.DYNAMIC, quadraticDrag=k), position=(0, 0, 0))
    st = _run(w, 1.0 / 240.0, 6000)
    assert abs(st['linear_velocity'][i][1]) == pytest.approx(math.sqrt(g / k), rel=1e-2)


# -- narrowphase primitives (test_collide_primitives.py) -------------------------
def _call(fn, *args, n=4):
    import ctypes as C
    ptr = C.POINTER(C.c_double)
    nrm, pts, dep = np.zeros(3), np.zeros(3 * n), np.zeros(n)
    conv = [C.c_double(a) if isinstance(a, float) else np.ascontiguousarray(a, 'd').ctypes.data_as(ptr)
            for a in args]
    k = fn(*conv, nrm.ctypes.data_as(ptr), pts.ctypes.data_as(ptr), dep.ctypes.data_as(ptr))
    return k, nrm, pts[:3 * k].reshape(-1, 3), dep[:k]


def _quat_matrix(q):
    R = np.zeros(9)
    import ctypes as C
    ptr = C.POINTER(C.c_double)
    q = np.ascontiguousarray(q, 'd')
    pyoracle.lib().or_quat_to_matrix(q.ctypes.data_as(ptr), R.ctypes.data_as(ptr))
    return R


def test_sphere_sphere_hit_and_miss():
    L = pyoracle.lib()
    k, n, p, d = _call(L.or_sphere_sphere, (0, 0, 0), 1.0, (1.5, 0, 0), 1.0)
    assert k == 1 and d[0] == pytest.approx(0.5) and np.allclose(n, (1, 0, 0)) and p[0][0] == pytest.approx(0.75)
    assert _call(L.or_sphere_sphere, (0, 0, 0), 1.0, (3, 0, 0), 1.0)[0] == 0


def test_sphere_box_face_miss_and_inside():
    L = pyoracle.lib()
    I3 = np.eye(3).reshape(9)
    k, n, _, d = _call(L.or_sphere_box, (0, 1.3, 0), 0.5, (0, 0, 0), I3, (1, 1, 1))
    assert k == 1 and d[0] == pytest.approx(0.2, abs=1e-9) and np.allclose(n, (0, -1, 0), atol=1e-9)
    assert _call(L.or_sphere_box, (0, 2.0, 0), 0.5, (0, 0, 0), I3, (1, 1, 1))[0] == 0
    k, n, _, _ = _call(L.or_sphere_box, (0.1, 0.0, 0.0), 0.2, (0, 0, 0), I3, (1, 0.3, 1))
    assert k == 1 and abs(n[1]) == pytest.approx(1.0)


def test_box_box_cases():
    L = pyoracle.lib()
    I3 = np.eye(3).reshape(9)
    k, n, _, d = _call(L.or_box_box, (0, 0, 0), I3, (1, 1, 1), (1.5, 0, 0), I3, (1, 1, 1))
    assert k > 0 and np.allclose(np.abs(n), (1, 0, 0), atol=1e-6) and max(d) == pytest.approx(0.5, abs=1e-6)
    k, n, _, _ = _call(L.or_box_box, (0, 0, 0), I3, (5, 0.5, 5), (0, 0.99, 0), I3, (0.5, 0.5, 0.5))
    assert k >= 3 and np.allclose(np.abs(n), (0, 1, 0), atol=1e-6)
    assert _call(L.or_box_box, (0, 0, 0), I3, (1, 1, 1), (3, 0, 0), I3, (1, 1, 1))[0] == 0
    s = math.sin(math.pi / 8)
    R = _quat_matrix((0.0, s, 0.0, math.cos(math.pi / 8)))
    assert _call(L.or_box_box, (0, 0, 0), I3, (1, 1, 1), (2.2, 0, 0), R, (1, 1, 1))[0] > 0


# -- solver (test_solver.py) ----------------------------------------------------------
DT = 1.0 / 120.0


def _ground(gravity_dir=(0, -1, 0), g=9.81, restitution=0.0, friction=0.6):
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=g, direction=gravity_dir), sleep_enabled=False)
    mat = w.add_material(M.Material(staticFriction=friction, dynamicFriction=friction, restitution=restitution))
    w.add_body(M.Motion(type=M.STATIC), M.Collider(shape=w.add_shape(M.Shape.box((40, 1, 40))), physicsMaterial=mat),
               position=(0, -0.5, 0))
    return w, mat


def _sphere(w, mat, height, radius=0.5):
    return w.add_body(M.Motion(type=M.DYNAMIC, mass=1.0),
                      M.Collider(shape=w.add_shape(M.Shape.sphere(radius)), physicsMaterial=mat),
                      position=(0, height, 0))


def test_no_restitution_comes_to_rest():
    w, mat = _ground(restitution=0.0)
    i = _sphere(w, mat, 3.0)
    st = _run(w, DT, 600)
    assert st['position'][i][1] == pytest.approx(0.5, abs=0.05) and abs(st['linear_velocity'][i][1]) < 0.2


def test_full_restitution_bounces_back_high():
    w, mat = _ground(restitution=1.0)
    i = _sphere(w, mat, 3.0)
    o = pyoracle.OracleWorld.from_world(w)
    bounced, peak = False, 0.0
    for _ in range(400):
        o.step(DT)
        y = o.state()['position'][i][1]
        if y < 0.6:
            bounced = True
        elif bounced:
            peak = max(peak, y)
    assert bounced and peak > 0.75 * 3.0


def test_resting_stack_is_stable():
    w, mat = _ground(restitution=0.0)
    shape = w.add_shape(M.Shape.box((1, 1, 1)))
    bodies = [w.add_body(M.Motion(type=M.DYNAMIC, mass=1.0), M.Collider(shape=shape, physicsMaterial=mat),
                         position=(0, 0.5 + k * 1.001, 0)) for k in range(5)]
    p = _run(w, DT, 600)['position']
    assert list(np.argsort([p[b][1] for b in bodies])) == [0, 1, 2, 3, 4]
    for k, b in enumerate(bodies):
        assert p[b][1] == pytest.approx(0.5 + k, abs=0.2) and abs(p[b][0]) < 0.5 and abs(p[b][2]) < 0.5


@pytest.mark.parametrize('angle_deg,friction,should_slide', [(40, 0.5, True), (10, 0.5, False)])
def test_incline_slides_iff_tan_exceeds_friction(angle_deg, friction, should_slide):
    t = math.radians(angle_deg)
    w, mat = _ground(gravity_dir=(math.sin(t), -math.cos(t), 0.0), friction=friction)
    i = w.add_body(M.Motion(type=M.DYNAMIC, mass=1.0),
                   M.Collider(shape=w.add_shape(M.Shape.box((1, 1, 1))), physicsMaterial=mat), position=(0, 0.5, 0))
    slid = _run(w, DT, 400)['position'][i][0]
    assert (slid > 0.5) if should_slide else (slid < 0.05)


def test_determinism_bit_identical_runs():
    def run():
        w, mat = _ground(restitution=0.3)
        shape = w.add_shape(M.Shape.box((1, 1, 1)))
        for k in range(6):
            w.add_body(M.Motion(type=M.DYNAMIC, mass=1.0), M.Collider(shape=shape, physicsMaterial=mat),
                       position=(0.3 * k, 1.0 + 1.2 * k, 0.1 * k))
        return _run(w, DT, 200)['position']
    assert np.array_equal(run(), run())


# -- gravity volumes (test_gravity.py) ------------------------------------------------
G = API.gravity


def test_point_gravity_pulls_body_toward_center():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=0.0))
    w.add_gravity_volume(G.GravityVolume(M.Gravity(type=M.POINT, gravity=9.81, center=(0, 0, 0)),
                                         G.SphereRegion((0, 0, 0), 100.0)))
    i = w.add_body(M.Motion(type=M.DYNAMIC), position=(10, 0, 0))
    st = _run(w, DT, 120)
    assert st['position'][i][0] < 10.0 and st['linear_velocity'][i][0] < 0


def test_higher_priority_replace_overrides_global():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=9.81, direction=(0, -1, 0)))
    w.add_gravity_volume(G.GravityVolume(M.Gravity(type=M.DIRECTIONAL, gravity=9.81, direction=(0, 1, 0),
                                                   priority=5, replace=True), G.SphereRegion((0, 0, 0), 100.0)))
    i = w.add_body(M.Motion(type=M.DYNAMIC), position=(0, 0, 0))
    assert _run(w, DT, 120)['linear_velocity'][i][1] > 0


def test_stop_zone_halts_gravity_accumulation():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=9.81, direction=(0, -1, 0)))
    w.add_gravity_volume(G.GravityVolume(M.Gravity(gravity=0.0, priority=5, stop=True), G.SphereRegion((0, 0, 0), 100.0)))
    i = w.add_body(M.Motion(type=M.DYNAMIC), position=(0, 0, 0))
    assert np.allclose(_run(w, DT, 120)['linear_velocity'][i], 0.0)


def test_region_bounds_limit_effect():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=0.0))
    w.add_gravity_volume(G.GravityVolume(M.Gravity(type=M.DIRECTIONAL, gravity=9.81, direction=(0, -1, 0)),
                                         G.SphereRegion((0, 0, 0), 1.0)))
    inside = w.add_body(M.Motion(type=M.DYNAMIC), position=(0, 0, 0))
    outside = w.add_body(M.Motion(type=M.DYNAMIC), position=(50, 0, 0))
    st = _run(w, DT, 120)
    assert st['linear_velocity'][inside][1] < -1.0 and np.allclose(st['linear_velocity'][outside], 0.0)


# -- sensors (test_triggers.py) -------------------------------------------------------
def _zone_world(zone_size, ball_radius, velocity, position):
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=0.0))
    w.add_body(M.Motion(type=M.STATIC), trigger=M.Trigger(shape=w.add_shape(M.Shape.box(zone_size))),
               position=(0, 0, 0))
    ball = w.add_body(M.Motion(type=M.DYNAMIC, linearVelocity=velocity),
                      M.Collider(shape=w.add_shape(M.Shape.sphere(ball_radius))), position=position)
    return w, ball


def _events(w, steps, dt=1.0 / 60.0):
    """Enter / stay / exit kinds per step, formed from the oracle's overlaps
    as the reference forms them (triggers.py:36-42)."""
    o = pyoracle.OracleWorld.from_world(w)
    prev, kinds = set(), []
    for _ in range(steps):
        o.step(dt)
        new = o.overlaps()
        kinds += ['enter'] * len(new - prev) + ['stay'] * len(new & prev) + ['exit'] * len(prev - new)
        prev = new
    return kinds, o.state()


def test_body_passing_through_trigger_fires_enter_and_exit():
    w, _ = _zone_world((1, 1, 1), 0.2, (2.0, 0, 0), (-3.0, 0, 0))
    kinds, _ = _events(w, 120)
    assert 'enter' in kinds and 'exit' in kinds and kinds.index('enter') < kinds.index('exit')


def test_trigger_does_not_perturb_trajectory():
    w, ball = _zone_world((1, 1, 1), 0.3, (2.0, 0, 0), (-3.0, 0, 0))
    _, st = _events(w, 120)
    assert np.allclose(st['linear_velocity'][ball], (2.0, 0, 0))
    assert st['position'][ball][1] == pytest.approx(0.0, abs=1e-9) and st['position'][ball][2] == pytest.approx(0.0, abs=1e-9)


def test_stay_events_while_inside():
    w, _ = _zone_world((2, 2, 2), 0.2, (0.0, 0.0, 0.0), (0, 0, 0))
    kinds, _ = _events(w, 5)
    assert kinds[0] == 'enter' and kinds.count('stay') >= 3


# -- joints (test_joints.py) ----------------------------------------------------------
JN = API.joints


def test_distance_constraint_keeps_pendulum_arm_length():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=9.81, direction=(0, -1, 0)), sleep_enabled=False)
    pivot = np.array([0.0, 5.0, 0.0])
    bob = w.add_body(M.Motion(type=M.DYNAMIC, mass=1.0), position=(2.0, 5.0, 0.0))
    w.add_joint_constraint(JN.DistanceConstraint(-1, bob, tuple(pivot), (0, 0, 0), 2.0))
    o = pyoracle.OracleWorld.from_world(w)
    lengths, lowest = [], 5.0
    for _ in range(600):
        o.step(DT)
        p = o.state()['position'][bob]
        lengths.append(np.linalg.norm(p - pivot))
        lowest = min(lowest, p[1])
    assert max(lengths) == pytest.approx(2.0, abs=0.05) and min(lengths) == pytest.approx(2.0, abs=0.05)
    assert lowest < 3.3


def test_point_constraint_pins_extended_body_at_offset():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=9.81, direction=(0, -1, 0)), sleep_enabled=False)
    bar = w.add_body(M.Motion(type=M.DYNAMIC, mass=1.0), M.Collider(shape=w.add_shape(M.Shape.box((2, 0.4, 0.4)))),
                     position=(1.0, 5.0, 0.0))
    w.add_joint_constraint(JN.PointConstraint(-1, bar, (0.0, 5.0, 0.0)))
    st = _run(w, DT, 400)
    R = _quat_matrix(st['orientation'][bar]).reshape(3, 3)
    assert np.allclose(st['position'][bar] + R @ np.array([-1.0, 0.0, 0.0]), (0.0, 5.0, 0.0), atol=0.05)
    assert st['position'][bar][1] < 4.9


def test_distance_constraint_holds_between_two_bodies():
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=9.81, direction=(0, -1, 0)), sleep_enabled=False)
    anchor = w.add_body(M.Motion(type=M.STATIC), position=(0, 5, 0))
    hanging = w.add_body(M.Motion(type=M.DYNAMIC, mass=1.0), position=(0, 2, 0))
    w.add_joint_constraint(JN.DistanceConstraint(anchor, hanging, (0, 0, 0), (0, 0, 0), 3.0))
    p = _run(w, DT, 600)['position']
    assert np.linalg.norm(p[hanging] - p[anchor]) == pytest.approx(3.0, abs=0.05)


def _spinner(target, max_force, steps):
    w = API.PhysicsWorld(gravity=M.Gravity(gravity=0.0), sleep_enabled=False)
    i = w.add_body(M.Motion(type=M.DYNAMIC, mass=1.0), M.Collider(shape=w.add_shape(M.Shape.box((1, 1, 1)))),
                   position=(0, 0, 0))
    w.add_joint_constraint(JN.AngularMotor(i, (0, 1, 0), target, max_force=max_force))
    return _run(w, DT, steps)['angular_velocity'][i]


def test_angular_motor_reaches_velocity_target():
    assert _spinner(3.0, 50.0, 240)[1] == pytest.approx(3.0, abs=0.1)


def test_motor_force_limit_caps_spin_up():
    assert _spinner(100.0, 0.5, 1)[1] < 5.0


# -- broadphase (test_broadphase.py) ----------------------------------------------------
@pytest.mark.parametrize('seed,spread', [(1, 3.0), (2, 6.0), (3, 1.5)])
def test_sweep_pairs_match_brute_force(seed, spread):
    """The oracle's sweep-and-prune pairs equal the O(N^2) overlap set over the
    same AABBs: boxes (>=, closed intervals) overlapping on all three axes, at
    least one dynamic body, interacting filters (broadphase.py:300-316)."""
    rng = np.random.default_rng(seed)
    w = API.PhysicsWorld()
    f_a = w.add_filter(M.CollisionFilter(collisionSystems=('a',), notCollideWithSystems=('b',)))
    f_b = w.add_filter(M.CollisionFilter(collisionSystems=('b',)))
    filters = (-1, f_a, f_b)
    for k in range(150):
        kind = (M.STATIC, M.KINEMATIC, M.DYNAMIC, M.DYNAMIC)[k % 4]
        shape = w.add_shape(M.Shape.sphere(0.5) if k % 3 else M.Shape.box(tuple(float(v) for v in rng.uniform(0.4, 1.2, 3))))
        w.add_body(M.Motion(type=kind), M.Collider(shape=shape, collisionFilter=filters[k % 3]),
                   position=tuple(float(v) for v in rng.uniform(-spread, spread, 3)), orientation=_quat_any(rng))
    o = pyoracle.OracleWorld.from_world(w)
    o.refit()
    got = {tuple(map(int, p)) for p in o.broadphase()}
    st = o.state()
    lo, hi = st['aabb_min'], st['aabb_max']
    mt = np.asarray(w._motion_type[:w.body_count])
    fl = np.asarray(w._collider_filter[:w.body_count])
    brute = set()
    for i in range(w.body_count):
        for j in range(i + 1, w.body_count):
            if mt[i] != 2 and mt[j] != 2:
                continue
            if not (np.all(hi[i] >= lo[j]) and np.all(hi[j] >= lo[i])):
                continue
            if w.filter_for(fl[i]).collides_with(w.filter_for(fl[j])):
                brute.add((i, j))
    assert got == brute and len(brute) > 0


def _quat_any(rng):
    q = rng.normal(size=4)
    return tuple(float(v) for v in q / np.linalg.norm(q))
