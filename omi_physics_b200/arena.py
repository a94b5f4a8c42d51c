"""Pack world objects into the library's arena tables (``OmiScene``).

Accepts any world with the reference's ``PhysicsWorld`` layout — the
reference's own class (``src/omi_physics/world.py``) or
:class:`omi_physics_b200.PhysicsWorld` — and concatenates one or more of
them. Indices become global (world offset added); ``-1`` keeps its meaning.
What the device path does not implement is refused here with
:class:`UnsupportedFeature`, never approximated.
"""
import ctypes as C
from typing import Sequence

import numpy as np

from ._lib import D, I, U8, OmiScene, UnsupportedFeature, WF_ACTIVE, WF_COLLISION, WF_SLEEP, \
    WF_WARM, ptr
from .gravity import pack_volumes
from .joints import joint_kind
from .model import COMBINE_CODES

# a cylinder is collided as a capsule (make_proxy, body.py:224-228)
SHAPE_CODES = {'sphere': 1, 'box': 2, 'convex': 3, 'capsule': 4, 'cylinder': 4, 'trimesh': 5}


def _quat_matrix(q) -> np.ndarray:
    """mathutil.quat_to_matrix (mathutil.py:59-76) of one quaternion, in numpy."""
    q = np.asarray(q, dtype='d')
    q = q / np.maximum(np.linalg.norm(q, axis=-1, keepdims=True), 1e-12)
    x, y, z, w = q[0], q[1], q[2], q[3]
    xx, yy, zz, xy, xz, yz, wx, wy, wz = x * x, y * y, z * z, x * y, x * z, y * z, w * x, w * y, w * z
    return np.array([[1 - 2 * (yy + zz), 2 * (xy - wz), 2 * (xz + wy)],
                     [2 * (xy + wz), 1 - 2 * (xx + zz), 2 * (yz - wx)],
                     [2 * (xz - wy), 2 * (yz + wx), 1 - 2 * (xx + yy)]])


def mesh_tables(points, indices, position, orientation) -> dict:
    """A mesh body's triangles as the reference collides them at this pose: world
    vertices (``points @ R.T + position``, body.py:164), per-triangle bounds
    and the uniform grid of trigrid.py:63-97 (64 cells along the longest
    side, triangles spanning more than 64 cells set aside, no grid below 256
    triangles), with numpy's arithmetic throughout."""
    R = _quat_matrix(orientation)
    wp = np.asarray(points, dtype='d') @ R.T + np.asarray(position, dtype='d')
    tris = wp[np.asarray(indices, dtype=np.int64).reshape(-1, 3)]
    lo, hi = tris.min(axis=1), tris.max(axis=1)
    T = len(tris)
    gi = np.zeros(4, np.int32)
    gd = np.zeros(7)
    cells = np.zeros((T, 6), np.int32)
    big = np.zeros(T, np.uint8)
    if T < 256:
        gi[0] = 1
    else:
        low, high = lo.min(axis=0), hi.max(axis=0)
        extent = np.maximum(high - low, 1e-9)
        cell = float(extent.max()) / 64
        top = (1 << 30) - 1
        first = np.clip(np.floor((lo - low) / cell).astype(int), 0, top)
        last = np.clip(np.floor((hi - low) / cell).astype(int), 0, top)
        gi[1:] = last.max(axis=0) + 1
        gd[:3], gd[3:6], gd[6] = low, high, cell
        cells[:, :3], cells[:, 3:] = first, last
        big[:] = np.prod(last - first + 1, axis=1) > 64
    return dict(verts=tris.reshape(T, 9), box=np.concatenate([lo, hi], axis=1), cells=cells, big=big,
                grid_i=gi, grid_d=gd, idx=np.asarray(indices, dtype=np.int32).reshape(-1, 3))
JOINT_CODES = {'point': 0, 'distance': 1, 'motor': 2}


def resolved_gravity(world) -> np.ndarray:
    """The uniform gravity vector exactly as ``resolve_gravity`` forms it (world.py:386-392)."""
    base = np.asarray(world.gravity.direction, dtype='d')
    norm = np.linalg.norm(base)
    base = base / norm if norm else base
    return base * world.gravity.gravity


def world_solver(world):
    col = getattr(world, '_collision', None)
    return getattr(col, 'solver', None) if col is not None else None


def world_flags(world, active: bool = True) -> int:
    solver = world_solver(world)
    f = 0
    if world.sleep_enabled:
        f |= WF_SLEEP
    if getattr(solver, 'warm_start', True):
        f |= WF_WARM
    if getattr(world, '_collision', None) is not None:
        f |= WF_COLLISION
    if active:
        f |= WF_ACTIVE
    return f


def world_iterations(world) -> int:
    solver = world_solver(world)
    return int(getattr(solver, 'velocity_iterations', 10)) if solver is not None else 10


def check_supported(world) -> None:
    """Raise :class:`UnsupportedFeature` for anything outside the device step."""
    n = world.body_count
    try:
        pack_volumes(getattr(world, 'gravity_volumes', None) or [])
    except (ValueError, AttributeError, TypeError) as e:
        raise UnsupportedFeature(-3, 'gravity volume outside the device path: %s' % e)
    used = set()
    for col in ('_collider_shape', '_trigger_shape'):
        cs = np.asarray(getattr(world, col)[:n])
        used |= set(int(s) for s in cs[(cs >= 0) & (cs < len(world.shapes))])
    for s in used:
        t = world.shapes[s].type
        if t not in SHAPE_CODES:
            raise UnsupportedFeature(-3, 'shape type %r is not supported on the CUDA path' % t)
    meshes = [k for k, sh in enumerate(world.shapes) if sh.type == 'trimesh']
    if meshes:
        ts = np.asarray(world._trigger_shape[:n])
        cs = np.asarray(world._collider_shape[:n])
        if np.isin(ts, meshes).any():
            raise UnsupportedFeature(-3, 'triangle-mesh sensors are not supported on the CUDA path')
        on = np.isin(cs, meshes)
        if (np.asarray(world._motion_type[:n])[on] == 2).any():
            raise UnsupportedFeature(-3, 'triangle meshes are taken as static or kinematic colliders only')
        for k in set(int(x) for x in cs[on]):
            if world.shapes[k].points is None or world.shapes[k].indices is None:
                raise UnsupportedFeature(-3, 'a triangle mesh needs its points and indices')


class PackedScene:
    """Numpy arrays behind one ``OmiScene`` (kept alive with it)."""

    def __init__(self):
        self.arrays = {}
        self.scene = OmiScene()

    def set(self, name, arr, t):
        arr = np.ascontiguousarray(arr)
        self.arrays[name] = arr
        setattr(self.scene, name, ptr(arr, t))


def pack_worlds(worlds: Sequence, dts: Sequence[float] = None, active=True) -> PackedScene:
    """Concatenate ``worlds`` into one arena description."""
    W = len(worlds)
    if W == 0:
        raise ValueError('no worlds')
    dts = list(dts) if dts is not None else [w.fixed_dt for w in worlds]
    act = [active] * W if isinstance(active, bool) else list(active)
    cols_f3 = ('position', 'linear_velocity', 'angular_velocity', 'inv_inertia')
    parts = {k: [] for k in ('pos', 'q', 'v', 'w', 'inv_mass', 'inv_inertia', 'gravity_factor',
                             'lin_damp', 'ang_damp', 'quad_drag', 'sleep_timer', 'motion_type',
                             'shape', 'material', 'material_key', 'filter_row', 'awake',
                             'shape_type', 'shape_radius', 'shape_size', 'shape_pt_off',
                             'shape_pt_cnt', 'points', 'mat_dynf', 'mat_rest', 'mat_fcomb',
                             'mat_rcomb', 'pf_a', 'pf_b', 'pf_mu', 'filter_matrix', 'j_type',
                             'j_a', 'j_b', 'j_anchor', 'j_anchor_b', 'j_local_a', 'j_local_b',
                             'j_has_local_a', 'j_has_local_b', 'j_length', 'j_has_length',
                             'j_axis', 'j_target', 'j_max_force', 'j_accum', 'trigger_shape',
                             'vol_kind', 'vol_g', 'vol_field', 'vol_rc', 'vol_rr', 'mesh_body',
                             'mesh_grid_i', 'mesh_grid_d', 'tri_verts', 'tri_box', 'tri_cells', 'tri_big',
                             'tri_idx')}
    body_off, joint_off, vol_off, tri_off = [0], [0], [0], [0]
    any_sensor = False
    w_g, w_dt, w_iters, w_jiters, w_flags, w_damp, w_solver = [], [], [], [], [], [], []
    w_foff, w_frows, w_pfoff, w_pfn = [], [], [], []
    nb = ns = nm = npts = nf = npf = nj = 0
    for wi, world in enumerate(worlds):
        check_supported(world)
        n = world.body_count
        parts['pos'].append(np.asarray(world._position[:n], 'd'))
        parts['q'].append(np.asarray(world._orientation[:n], 'd'))
        parts['v'].append(np.asarray(world._linear_velocity[:n], 'd'))
        parts['w'].append(np.asarray(world._angular_velocity[:n], 'd'))
        parts['inv_mass'].append(np.asarray(world._inv_mass[:n], 'd'))
        parts['inv_inertia'].append(np.asarray(world._inv_inertia[:n], 'd'))
        parts['gravity_factor'].append(np.asarray(world._gravity_factor[:n], 'd'))
        parts['lin_damp'].append(np.asarray(world._linear_damping[:n], 'd'))
        parts['ang_damp'].append(np.asarray(world._angular_damping[:n], 'd'))
        parts['quad_drag'].append(np.asarray(world._quadratic_drag[:n], 'd'))
        parts['sleep_timer'].append(np.asarray(world._sleep_timer[:n], 'd'))
        parts['motion_type'].append(np.asarray(world._motion_type[:n], np.int32))
        parts['awake'].append(np.asarray(world._awake[:n], np.uint8))
        cs = np.asarray(world._collider_shape[:n], np.int64)
        valid = (cs >= 0) & (cs < len(world.shapes))
        parts['shape'].append(np.where(valid, cs + ns, -1).astype(np.int32))
        ts = np.asarray(world._trigger_shape[:n], np.int64)
        tvalid = (ts >= 0) & (ts < len(world.shapes))
        any_sensor |= bool(tvalid.any())
        parts['trigger_shape'].append(np.where(tvalid, ts + ns, -1).astype(np.int32))
        for i in range(n):
            if valid[i] and world.shapes[int(cs[i])].type == 'trimesh':
                sh = world.shapes[int(cs[i])]
                mt = mesh_tables(sh.points, sh.indices, world._position[i], world._orientation[i])
                parts['mesh_body'].append([nb + i])
                parts['mesh_grid_i'].append(mt['grid_i'])
                parts['mesh_grid_d'].append(mt['grid_d'])
                for key in ('verts', 'box', 'cells', 'big', 'idx'):
                    parts['tri_' + key].append(mt[key])
                tri_off.append(tri_off[-1] + len(mt['big']))
        vols = pack_volumes(getattr(world, 'gravity_volumes', None) or [])
        for key in ('kind', 'g', 'field', 'rc', 'rr'):
            if len(vols[key]):
                parts['vol_' + key].append(vols[key])
        vol_off.append(vol_off[-1] + len(vols['kind']))
        cm = np.asarray(world._collider_material[:n], np.int64)
        mvalid = (cm >= 0) & (cm < len(world.materials))
        parts['material'].append(np.where(mvalid, cm + nm, -1).astype(np.int32))
        parts['material_key'].append(cm.astype(np.int32))
        cf = np.asarray(world._collider_filter[:n], np.int64)
        F = len(world.filters)
        parts['filter_row'].append(np.where((cf >= 0) & (cf < F), cf + 1, 0).astype(np.int32))
        # shapes
        for sh in world.shapes:
            code = SHAPE_CODES.get(sh.type, 0)
            parts['shape_type'].append([code])
            if code == 4:
                # capsule proxy: radiusBottom, half height 0.5 * height
                parts['shape_radius'].append([float(sh.radiusBottom)])
                parts['shape_size'].append(np.array([[0.0, float(sh.height), 0.0]]))
            else:
                parts['shape_radius'].append([float(sh.radius)])
                size = np.asarray(sh.size, 'd') if np.size(sh.size) == 3 else np.zeros(3)
                parts['shape_size'].append(size.reshape(1, 3))
            if sh.type in ('convex', 'trimesh') and sh.points is not None:
                pts = np.asarray(sh.points, 'd').reshape(-1, 3)
                parts['shape_pt_off'].append([npts])
                parts['shape_pt_cnt'].append([len(pts)])
                parts['points'].append(pts)
                npts += len(pts)
            else:
                parts['shape_pt_off'].append([0])
                parts['shape_pt_cnt'].append([0])
        # materials
        for m in world.materials:
            parts['mat_dynf'].append([m.dynamicFriction])
            parts['mat_rest'].append([m.restitution])
            parts['mat_fcomb'].append([COMBINE_CODES.get(m.frictionCombine, 0)])
            parts['mat_rcomb'].append([COMBINE_CODES.get(m.restitutionCombine, 0)])
        pf = sorted(world.pair_friction.items())
        w_pfoff.append(npf)
        w_pfn.append(len(pf))
        for (ka, kb), (_, mu) in pf:
            parts['pf_a'].append([ka]); parts['pf_b'].append([kb]); parts['pf_mu'].append([mu])
        npf += len(pf)
        # filter matrix, row 0 = default filter
        flist = [world.filter_for(-1)] + list(world.filters)
        fm = np.array([[1 if a.collides_with(b) else 0 for b in flist] for a in flist], np.uint8)
        w_foff.append(nf)
        w_frows.append(F + 1)
        parts['filter_matrix'].append(fm.reshape(-1))
        nf += fm.size
        # joints
        js = list(world.joint_constraints)
        for c in js:
            k = joint_kind(c)
            parts['j_type'].append([JOINT_CODES[k]])
            z3 = np.zeros((1, 3))
            if k == 'motor':
                parts['j_a'].append([c.body + nb]); parts['j_b'].append([-1])
                parts['j_anchor'].append(z3); parts['j_anchor_b'].append(z3)
                parts['j_local_a'].append(z3); parts['j_local_b'].append(z3)
                parts['j_has_local_a'].append([0]); parts['j_has_local_b'].append([0])
                parts['j_length'].append([0.0]); parts['j_has_length'].append([0])
                parts['j_axis'].append(np.asarray(c.axis, 'd').reshape(1, 3))
                parts['j_target'].append([c.target]); parts['j_max_force'].append([c.max_force])
                parts['j_accum'].append([c.accum])
                continue
            parts['j_a'].append([c.a + nb if c.a >= 0 else -1])
            parts['j_b'].append([c.b + nb if c.b >= 0 else -1])
            parts['j_axis'].append(z3); parts['j_target'].append([0.0])
            parts['j_max_force'].append([0.0]); parts['j_accum'].append([0.0])
            if k == 'point':
                parts['j_anchor'].append(np.asarray(c.anchor, 'd').reshape(1, 3))
                parts['j_anchor_b'].append(z3)
                for side, loc in (('a', c.local_a), ('b', c.local_b)):
                    has = loc is not None
                    parts['j_local_' + side].append(np.asarray(loc, 'd').reshape(1, 3) if has else z3)
                    parts['j_has_local_' + side].append([1 if has else 0])
                parts['j_length'].append([0.0]); parts['j_has_length'].append([0])
            else:
                parts['j_anchor'].append(np.asarray(c.anchor_a, 'd').reshape(1, 3))
                parts['j_anchor_b'].append(np.asarray(c.anchor_b, 'd').reshape(1, 3))
                parts['j_local_a'].append(z3); parts['j_local_b'].append(z3)
                parts['j_has_local_a'].append([0]); parts['j_has_local_b'].append([0])
                has = c.length is not None
                parts['j_length'].append([float(c.length) if has else 0.0])
                parts['j_has_length'].append([1 if has else 0])
        nj += len(js)
        joint_off.append(nj)
        # per-world parameters
        w_g.append(resolved_gravity(world))
        w_dt.append(float(dts[wi]))
        w_iters.append(world_iterations(world))
        w_jiters.append(int(world.joint_iterations))
        w_flags.append(world_flags(world, act[wi]))
        w_damp.append([world.default_linear_damping, world.default_angular_damping])
        solver = world_solver(world)
        w_solver.append([float(getattr(solver, 'restitution_threshold', 0.5)),
                         float(getattr(solver, 'slop', 0.005))])
        nb += n
        ns += len(world.shapes)
        nm += len(world.materials)
        body_off.append(nb)

    def cat(key, dtype, width=None):
        xs = parts[key]
        if not xs:
            shape = (1,) if width is None else (1, width)
            return np.zeros(shape, dtype)
        arrs = [np.asarray(x, dtype) for x in xs]
        if width is not None:
            arrs = [a.reshape(-1, width) for a in arrs]
            return np.concatenate(arrs, axis=0)
        return np.concatenate([a.reshape(-1) for a in arrs])

    P = PackedScene()
    s = P.scene
    s.n_worlds = W
    P.set('w_body_off', np.array(body_off, np.int32), I)
    P.set('w_gravity', np.array(w_g, 'd').reshape(W, 3), D)
    P.set('w_dt', np.array(w_dt, 'd'), D)
    P.set('w_iters', np.array(w_iters, np.int32), I)
    P.set('w_joint_iters', np.array(w_jiters, np.int32), I)
    P.set('w_flags', np.array(w_flags, np.int32), I)
    P.set('w_default_damp', np.array(w_damp, 'd').reshape(W, 2), D)
    P.set('w_solver', np.array(w_solver, 'd').reshape(W, 2), D)
    P.set('w_filter_off', np.array(w_foff, np.int32), I)
    P.set('w_filter_rows', np.array(w_frows, np.int32), I)
    P.set('w_pf_off', np.array(w_pfoff, np.int32), I)
    P.set('w_pf_n', np.array(w_pfn, np.int32), I)
    P.set('w_joint_off', np.array(joint_off, np.int32), I)
    s.n_bodies = nb
    for key, t, dt, width in (('pos', D, 'd', 3), ('q', D, 'd', 4), ('v', D, 'd', 3),
                              ('w', D, 'd', 3), ('inv_mass', D, 'd', None),
                              ('inv_inertia', D, 'd', 3), ('gravity_factor', D, 'd', None),
                              ('lin_damp', D, 'd', None), ('ang_damp', D, 'd', None),
                              ('quad_drag', D, 'd', None), ('sleep_timer', D, 'd', None),
                              ('motion_type', I, np.int32, None), ('shape', I, np.int32, None),
                              ('material', I, np.int32, None), ('material_key', I, np.int32, None),
                              ('filter_row', I, np.int32, None), ('awake', U8, np.uint8, None)):
        P.set(key, cat(key, dt, width), t)
    s.n_shapes = ns
    P.set('shape_type', cat('shape_type', np.int32), I)
    P.set('shape_radius', cat('shape_radius', 'd'), D)
    P.set('shape_size', cat('shape_size', 'd', 3), D)
    P.set('shape_pt_off', cat('shape_pt_off', np.int32), I)
    P.set('shape_pt_cnt', cat('shape_pt_cnt', np.int32), I)
    s.n_points = npts
    P.set('points', cat('points', 'd', 3), D)
    s.n_materials = nm
    P.set('mat_dynf', cat('mat_dynf', 'd'), D)
    P.set('mat_rest', cat('mat_rest', 'd'), D)
    P.set('mat_fcomb', cat('mat_fcomb', np.int32), I)
    P.set('mat_rcomb', cat('mat_rcomb', np.int32), I)
    s.n_pair_friction = npf
    P.set('pf_a', cat('pf_a', np.int32), I)
    P.set('pf_b', cat('pf_b', np.int32), I)
    P.set('pf_mu', cat('pf_mu', 'd'), D)
    s.n_filter_bytes = nf
    P.set('filter_matrix', cat('filter_matrix', np.uint8), U8)
    s.n_joints = nj
    for key, t, dt, width in (('j_type', I, np.int32, None), ('j_a', I, np.int32, None),
                              ('j_b', I, np.int32, None), ('j_anchor', D, 'd', 3),
                              ('j_anchor_b', D, 'd', 3), ('j_local_a', D, 'd', 3),
                              ('j_local_b', D, 'd', 3), ('j_has_local_a', U8, np.uint8, None),
                              ('j_has_local_b', U8, np.uint8, None), ('j_length', D, 'd', None),
                              ('j_has_length', U8, np.uint8, None), ('j_axis', D, 'd', 3),
                              ('j_target', D, 'd', None), ('j_max_force', D, 'd', None),
                              ('j_accum', D, 'd', None)):
        P.set(key, cat(key, dt, width), t)
    if any_sensor:
        P.set('trigger_shape', cat('trigger_shape', np.int32), I)
    if vol_off[-1]:
        P.set('w_vol_off', np.array(vol_off, np.int32), I)
        s.n_volumes = vol_off[-1]
        P.set('vol_kind', cat('vol_kind', np.int32), I)
        P.set('vol_g', cat('vol_g', 'd'), D)
        for key in ('vol_field', 'vol_rc', 'vol_rr'):
            P.set(key, cat(key, 'd', 3), D)
    if len(tri_off) > 1:
        s.n_meshes = len(tri_off) - 1
        P.set('mesh_body', cat('mesh_body', np.int32), I)
        P.set('mesh_tri_off', np.array(tri_off, np.int32), I)
        P.set('mesh_grid_i', cat('mesh_grid_i', np.int32, 4), I)
        P.set('mesh_grid_d', cat('mesh_grid_d', 'd', 7), D)
        P.set('tri_verts', cat('tri_verts', 'd', 9), D)
        P.set('tri_box', cat('tri_box', 'd', 6), D)
        P.set('tri_cells', cat('tri_cells', np.int32, 6), I)
        P.set('tri_big', cat('tri_big', np.uint8), U8)
        P.set('tri_idx', cat('tri_idx', np.int32, 3), I)
    P.has_sensors = any_sensor
    P.body_off = body_off
    P.joint_off = joint_off
    P.n_bodies = nb
    P.n_joints = nj
    P.worlds = list(worlds)
    return P


def static_signature(world) -> tuple:
    """What forces a re-pack when it changes: topology and the static columns."""
    import zlib
    n = world.body_count
    crc = 0
    for name in ('_inv_mass', '_inv_inertia', '_gravity_factor', '_linear_damping',
                 '_angular_damping', '_quadratic_drag', '_motion_type', '_collider_shape',
                 '_collider_material', '_collider_filter', '_trigger_shape'):
        crc = zlib.crc32(np.ascontiguousarray(getattr(world, name)[:n]).view(np.uint8), crc)
    vols = pack_volumes(getattr(world, 'gravity_volumes', None) or [])
    for key in ('kind', 'g', 'field', 'rc', 'rr'):
        crc = zlib.crc32(np.ascontiguousarray(vols[key]).view(np.uint8), crc)
    return (n, len(world.shapes), len(world.materials), len(world.filters),
            len(world.joint_constraints), tuple(sorted(world.pair_friction.items())),
            tuple(id(c) for c in world.joint_constraints), world.gravity.gravity,
            tuple(world.gravity.direction), len(vols['kind']), crc)
