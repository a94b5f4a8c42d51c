"""ctypes wrapper of the C oracle (test infrastructure only).

``OracleWorld.from_world(world)`` snapshots any world object that has the
reference's ``PhysicsWorld`` attribute layout (the reference's own class or
``omi_physics_b200.PhysicsWorld``) into the oracle's arrays; ``step()`` runs
``or_step`` (a CPU restatement of ``PhysicsWorld.step``, world.py:410-430) and
exposes the per-step pairs, contacts, impulses and sleep islands.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, always as the parity reference or the timed CPU baseline.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int32)
U8 = C.POINTER(C.c_uint8)


class OrWorldC(C.Structure):
    _fields_ = [
        ('n', C.c_int32),
        ('pos', D), ('q', D), ('v', D), ('w', D), ('prev_pos', D), ('prev_q', D),
        ('inv_mass', D), ('inv_inertia', D),
        ('gravity_factor', D), ('lin_damp', D), ('ang_damp', D), ('quad_drag', D),
        ('sleep_timer', D),
        ('motion_type', I), ('collider_shape', I), ('collider_material', I),
        ('collider_filter', I),
        ('awake', U8),
        ('aabb_min', D), ('aabb_max', D),
        ('n_shapes', C.c_int32), ('shape_type', I), ('shape_radius', D), ('shape_size', D),
        ('shape_pt_off', I), ('shape_pt_cnt', I), ('points', D),
        ('n_materials', C.c_int32), ('mat_dynf', D), ('mat_rest', D), ('mat_fcomb', I),
        ('mat_rcomb', I),
        ('n_pair_friction', C.c_int32), ('pf_a', I), ('pf_b', I), ('pf_mu', D),
        ('n_filters', C.c_int32), ('filter_matrix', U8),
        ('n_joints', C.c_int32), ('j_type', I), ('j_a', I), ('j_b', I),
        ('j_anchor', D), ('j_anchor_b', D), ('j_local_a', D), ('j_local_b', D),
        ('j_has_local_a', U8), ('j_has_local_b', U8), ('j_length', D), ('j_has_length', U8),
        ('j_axis', D), ('j_target', D), ('j_max_force', D), ('j_accum', D),
        ('g', C.c_double * 3), ('dt', C.c_double),
        ('default_lin_damp', C.c_double), ('default_ang_damp', C.c_double),
        ('velocity_iterations', C.c_int32), ('joint_iterations', C.c_int32),
        ('sleep_enabled', C.c_int32), ('warm_start', C.c_int32), ('has_collision', C.c_int32),
        ('restitution_threshold', C.c_double), ('slop', C.c_double),
        ('correction', C.c_double), ('margin', C.c_double),
        ('cache_n', C.c_int32), ('cache_a', I), ('cache_b', I), ('cache_pt', D),
        ('cache_imp', D),
        ('n_pairs', C.c_int32), ('n_solid', C.c_int32), ('pairs', I), ('solid', I),
        ('n_contacts', C.c_int32), ('c_a', I), ('c_b', I), ('c_pt', D), ('c_n', D),
        ('c_depth', D), ('c_imp', D),
        ('island', I),
        ('trigger_shape', I),
        ('n_volumes', C.c_int32), ('vol_kind', I), ('vol_g', D), ('vol_field', D), ('vol_rc', D),
        ('vol_rr', D),
        ('n_overlaps', C.c_int32), ('ov_trg', I), ('ov_other', I),
        ('shape_tri_off', I), ('shape_tri_cnt', I), ('tris', I),
    ]


def build():
    """Compile liboracle.so with oracle/Makefile (no FMA contraction)."""
    subprocess.run(['make', '-s', '-C', _HERE], check=True)


def lib():
    """Load (building if needed) the oracle library."""
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, 'liboracle.so')
        src = os.path.join(_HERE, 'oracle.c')
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = C.CDLL(path)
        L.or_step.argtypes = [C.POINTER(OrWorldC)]
        L.or_step.restype = C.c_int
        for name in ('or_refit', 'or_integrate_forces', 'or_integrate_positions', 'or_free'):
            getattr(L, name).argtypes = [C.POINTER(OrWorldC)]
            getattr(L, name).restype = None
        L.or_broadphase.argtypes = [C.POINTER(OrWorldC)]
        L.or_broadphase.restype = C.c_int
        L.or_set_cache.argtypes = [C.POINTER(OrWorldC), C.c_int32, I, I, D, D]
        L.or_set_cache.restype = C.c_int
        for name in ('or_box_box',):
            getattr(L, name).argtypes = [D, D, D, D, D, D, D, D, D]
            getattr(L, name).restype = C.c_int
        L.or_sphere_sphere.argtypes = [D, C.c_double, D, C.c_double, D, D, D]
        L.or_sphere_sphere.restype = C.c_int
        L.or_sphere_box.argtypes = [D, C.c_double, D, D, D, D, D, D]
        L.or_sphere_box.restype = C.c_int
        L.or_quat_to_matrix.argtypes = [D, D]
        L.or_quat_to_matrix.restype = None
        L.or_capsule_triangles.argtypes = [D, D, C.c_double, D, C.c_int64, U8, D, D, D]
        L.or_capsule_triangles.restype = None
        _LIB = L
    return _LIB


def _ptr(a, t):
    return a.ctypes.data_as(t)


# a cylinder is collided as a capsule by the reference (body.py:224-228)
SHAPE_CODES = {'sphere': 1, 'box': 2, 'convex': 3, 'capsule': 4, 'cylinder': 4, 'trimesh': 5}
COMBINE = {'average': 0, 'minimum': 1, 'maximum': 2, 'multiply': 3}
JOINT_CODES = {'point': 0, 'distance': 1, 'motor': 2}


def _pack_volumes(volumes):
    """The oracle's gravity-volume table (oracle.h): stable priority order
    (gravity.py:89); a directional field precomputed with numpy exactly as
    ``GravityVolume.field_at`` computes it (gravity.py:66-79); a sphere region's
    ``radius ** 2`` as gravity.py:25 evaluates it."""
    ordered = sorted(volumes, key=lambda v: v.priority)
    m = len(ordered)
    kind = np.zeros(max(m, 1), np.int32)
    g, field = np.zeros(max(m, 1)), np.zeros((max(m, 1), 3))
    rc, rr = np.zeros((max(m, 1), 3)), np.zeros((max(m, 1), 3))
    for k, v in enumerate(ordered):
        f = v.field
        if f.type == 'point':
            kind[k] |= 1
            field[k] = np.asarray(f.center, dtype='d')
        else:
            d = np.asarray(f.direction, dtype='d')
            field[k] = d / np.maximum(np.linalg.norm(d, axis=-1, keepdims=True), 1e-12) * f.gravity
        g[k] = f.gravity
        if f.replace:
            kind[k] |= 8
        elif f.stop:
            kind[k] |= 16
        reg = v.region
        name = type(reg).__name__
        if name == 'SphereRegion':
            kind[k] |= 2
            rc[k] = reg.center
            rr[k, 0] = reg.radius ** 2
        elif name == 'BoxRegion':
            kind[k] |= 4
            rc[k] = reg.center
            rr[k] = reg.half
        elif name != 'InfiniteRegion':
            raise ValueError('region %s' % name)
    return m, dict(vol_kind=kind, vol_g=g, vol_field=field, vol_rc=rc, vol_rr=rr)


def _joint_kind(c):
    k = getattr(c, 'kind', None)
    if k in JOINT_CODES:
        return k
    return {'PointConstraint': 'point', 'DistanceConstraint': 'distance',
            'AngularMotor': 'motor'}[type(c).__name__]


class OracleWorld:
    """Numpy-owned oracle state for one world."""

    def __init__(self):
        self.c = OrWorldC()
        self._keep = {}

    def _set(self, name, arr, t):
        self._keep[name] = arr
        setattr(self.c, name, _ptr(arr, t))

    @classmethod
    def from_world(cls, world, warm_start=None):
        """Snapshot ``world`` (reference-compatible layout) into oracle arrays."""
        self = cls()
        n = world.body_count
        c = self.c
        c.n = n
        f64 = lambda name, width=None: np.ascontiguousarray(
            getattr(world, '_' + name)[:n], dtype=np.float64).copy()
        for name, field, t in (('position', 'pos', D), ('orientation', 'q', D),
                               ('linear_velocity', 'v', D), ('angular_velocity', 'w', D),
                               ('prev_position', 'prev_pos', D),
                               ('prev_orientation', 'prev_q', D),
                               ('inv_mass', 'inv_mass', D), ('inv_inertia', 'inv_inertia', D),
                               ('gravity_factor', 'gravity_factor', D),
                               ('linear_damping', 'lin_damp', D),
                               ('angular_damping', 'ang_damp', D),
                               ('quadratic_drag', 'quad_drag', D),
                               ('sleep_timer', 'sleep_timer', D)):
            self._set(field, f64(name), t)
        for name in ('motion_type', 'collider_shape', 'collider_material', 'collider_filter'):
            self._set(name, np.ascontiguousarray(getattr(world, '_' + name)[:n], dtype=np.int32).copy(), I)
        self._set('awake', np.ascontiguousarray(world._awake[:n], dtype=np.uint8).copy(), U8)
        self._set('aabb_min', np.zeros((max(n, 1), 3)), D)
        self._set('aabb_max', np.zeros((max(n, 1), 3)), D)
        self._set('island', np.full(max(n, 1), -1, dtype=np.int32), I)
        ts = np.ascontiguousarray(getattr(world, '_trigger_shape')[:n], dtype=np.int32).copy()
        if n and np.any(ts >= 0):
            self._set('trigger_shape', ts, I)
        c.n_volumes, vols = _pack_volumes(getattr(world, 'gravity_volumes', None) or [])
        for name, arr in vols.items():
            self._set(name, arr, I if name == 'vol_kind' else D)
        # shapes
        shapes = world.shapes
        ns = len(shapes)
        stype = np.zeros(max(ns, 1), np.int32)
        srad = np.zeros(max(ns, 1))
        ssize = np.zeros((max(ns, 1), 3))
        poff = np.zeros(max(ns, 1), np.int32)
        pcnt = np.zeros(max(ns, 1), np.int32)
        pts = []
        total = 0
        toff = np.zeros(max(ns, 1), np.int32)
        tcnt = np.zeros(max(ns, 1), np.int32)
        tris = []
        ntri = 0
        for s, sh in enumerate(shapes):
            if sh.type not in SHAPE_CODES:
                stype[s] = 0
                continue
            stype[s] = SHAPE_CODES[sh.type]
            if stype[s] == 4:
                srad[s] = sh.radiusBottom
                ssize[s] = (0.0, float(sh.height), 0.0)
            else:
                srad[s] = sh.radius
                ssize[s] = np.asarray(sh.size, dtype='d')
            if sh.type in ('convex', 'trimesh') and sh.points is not None:
                p = np.asarray(sh.points, dtype='d').reshape(-1, 3)
                poff[s] = total
                pcnt[s] = len(p)
                total += len(p)
                pts.append(p)
            if sh.type == 'trimesh' and sh.indices is not None:
                t = np.asarray(sh.indices, dtype=np.int32).reshape(-1, 3)
                toff[s] = ntri
                tcnt[s] = len(t)
                ntri += len(t)
                tris.append(t)
        points = np.ascontiguousarray(np.concatenate(pts) if pts else np.zeros((1, 3)))
        c.n_shapes = ns
        self._set('shape_type', stype, I); self._set('shape_radius', srad, D)
        self._set('shape_size', ssize, D); self._set('shape_pt_off', poff, I)
        self._set('shape_pt_cnt', pcnt, I); self._set('points', points, D)
        self._set('shape_tri_off', toff, I); self._set('shape_tri_cnt', tcnt, I)
        self._set('tris', np.ascontiguousarray(np.concatenate(tris) if tris else np.zeros((1, 3), np.int32)), I)
        # materials
        mats = world.materials
        nm = len(mats)
        c.n_materials = nm
        self._set('mat_dynf', np.array([m.dynamicFriction for m in mats] or [0.0], dtype='d'), D)
        self._set('mat_rest', np.array([m.restitution for m in mats] or [0.0], dtype='d'), D)
        self._set('mat_fcomb', np.array([COMBINE.get(m.frictionCombine, 0) for m in mats] or [0], dtype=np.int32), I)
        self._set('mat_rcomb', np.array([COMBINE.get(m.restitutionCombine, 0) for m in mats] or [0], dtype=np.int32), I)
        pf = sorted(world.pair_friction.items())
        c.n_pair_friction = len(pf)
        self._set('pf_a', np.array([k[0] for k, _ in pf] or [0], dtype=np.int32), I)
        self._set('pf_b', np.array([k[1] for k, _ in pf] or [0], dtype=np.int32), I)
        self._set('pf_mu', np.array([v[1] for _, v in pf] or [0.0], dtype='d'), D)
        # filters: row 0 = default filter
        flist = [world.filter_for(-1)] + list(world.filters)
        nf = len(world.filters)
        fm = np.zeros((nf + 1, nf + 1), dtype=np.uint8)
        for i, fa in enumerate(flist):
            for j, fb in enumerate(flist):
                fm[i, j] = 1 if fa.collides_with(fb) else 0
        c.n_filters = nf
        self._set('filter_matrix', np.ascontiguousarray(fm), U8)
        # joints
        js = list(world.joint_constraints)
        self.joint_objs = js
        J = len(js)
        c.n_joints = J
        jt = np.zeros(max(J, 1), np.int32); ja = np.full(max(J, 1), -1, np.int32)
        jb = np.full(max(J, 1), -1, np.int32)
        anc = np.zeros((max(J, 1), 3)); ancb = np.zeros((max(J, 1), 3))
        la = np.zeros((max(J, 1), 3)); lb = np.zeros((max(J, 1), 3))
        hla = np.zeros(max(J, 1), np.uint8); hlb = np.zeros(max(J, 1), np.uint8)
        ln = np.zeros(max(J, 1)); hln = np.zeros(max(J, 1), np.uint8)
        ax = np.zeros((max(J, 1), 3)); tg = np.zeros(max(J, 1)); mf = np.zeros(max(J, 1))
        acc = np.zeros(max(J, 1))
        for j, o in enumerate(js):
            k = _joint_kind(o)
            jt[j] = JOINT_CODES[k]
            if k == 'motor':
                ja[j] = o.body
                ax[j] = o.axis; tg[j] = o.target; mf[j] = o.max_force; acc[j] = o.accum
            elif k == 'point':
                ja[j], jb[j] = o.a, o.b
                anc[j] = o.anchor
                if o.local_a is not None:
                    la[j] = o.local_a; hla[j] = 1
                if o.local_b is not None:
                    lb[j] = o.local_b; hlb[j] = 1
            else:
                ja[j], jb[j] = o.a, o.b
                anc[j] = o.anchor_a; ancb[j] = o.anchor_b
                if o.length is not None:
                    ln[j] = o.length; hln[j] = 1
        for name, arr, t in (('j_type', jt, I), ('j_a', ja, I), ('j_b', jb, I),
                             ('j_anchor', anc, D), ('j_anchor_b', ancb, D),
                             ('j_local_a', la, D), ('j_local_b', lb, D),
                             ('j_has_local_a', hla, U8), ('j_has_local_b', hlb, U8),
                             ('j_length', ln, D), ('j_has_length', hln, U8),
                             ('j_axis', ax, D), ('j_target', tg, D), ('j_max_force', mf, D),
                             ('j_accum', acc, D)):
            self._set(name, arr, t)
        # parameters
        base = np.asarray(world.gravity.direction, dtype='d')
        norm = np.linalg.norm(base)
        base = base / norm if norm else base
        g = base * world.gravity.gravity
        c.g = (C.c_double * 3)(*g)
        c.default_lin_damp = world.default_linear_damping
        c.default_ang_damp = world.default_angular_damping
        col = world._collision
        solver = getattr(col, 'solver', None) if col is not None else None
        c.has_collision = 1 if col is not None else 0
        c.velocity_iterations = int(getattr(solver, 'velocity_iterations', 10))
        c.joint_iterations = int(world.joint_iterations)
        c.sleep_enabled = 1 if world.sleep_enabled else 0
        ws = getattr(solver, 'warm_start', True) if warm_start is None else warm_start
        c.warm_start = 1 if ws else 0
        c.restitution_threshold = float(getattr(solver, 'restitution_threshold', 0.5))
        c.slop = float(getattr(solver, 'slop', 0.005))
        c.correction = 0.8
        c.margin = 0.05
        cache = getattr(solver, '_cache', None)
        if cache:
            self.set_cache_dict(cache)
        return self

    def set_cache_dict(self, cache):
        """Load a reference-style ``{(a, b): [(point, n, t0, t1), ...]}`` cache."""
        a, b, pt, imp = [], [], [], []
        for (i, j), entries in cache.items():
            for point, n, t0, t1 in entries:
                a.append(i); b.append(j); pt.append(point); imp.append((n, t0, t1))
        self.set_cache(np.array(a, np.int32), np.array(b, np.int32),
                       np.array(pt, 'd').reshape(-1, 3), np.array(imp, 'd').reshape(-1, 3))

    def set_cache(self, a, b, pt, imp):
        a = np.ascontiguousarray(a, np.int32); b = np.ascontiguousarray(b, np.int32)
        pt = np.ascontiguousarray(pt, 'd'); imp = np.ascontiguousarray(imp, 'd')
        rc = lib().or_set_cache(C.byref(self.c), len(a), _ptr(a, I), _ptr(b, I), _ptr(pt, D),
                                _ptr(imp, D))
        assert rc == 0

    def step(self, dt):
        self.c.dt = dt
        rc = lib().or_step(C.byref(self.c))
        if rc != 0:
            raise RuntimeError('oracle step failed: %d' % rc)

    def refit(self):
        lib().or_refit(C.byref(self.c))

    def broadphase(self):
        assert lib().or_broadphase(C.byref(self.c)) == 0
        return self.pairs()

    # -- outputs --------------------------------------------------------
    def _arr(self, ptr, n, shape, dtype):
        if n == 0:
            return np.zeros((0,) + shape[1:], dtype=dtype)
        return np.ctypeslib.as_array(ptr, shape=shape).copy()

    def pairs(self):
        return self._arr(self.c.pairs, self.c.n_pairs, (self.c.n_pairs, 2), np.int32)

    def solid_pairs(self):
        return self._arr(self.c.solid, self.c.n_solid, (self.c.n_solid, 2), np.int32)

    def contacts(self):
        K = self.c.n_contacts
        return dict(a=self._arr(self.c.c_a, K, (K,), np.int32),
                    b=self._arr(self.c.c_b, K, (K,), np.int32),
                    point=self._arr(self.c.c_pt, K, (K, 3), 'd'),
                    normal=self._arr(self.c.c_n, K, (K, 3), 'd'),
                    depth=self._arr(self.c.c_depth, K, (K,), 'd'),
                    impulse=self._arr(self.c.c_imp, K, (K, 3), 'd'))

    def overlaps(self):
        """This step's trigger overlaps as a set of (trigger, other) body pairs."""
        k = self.c.n_overlaps
        t = self._arr(self.c.ov_trg, k, (k,), np.int32)
        o = self._arr(self.c.ov_other, k, (k,), np.int32)
        return {(int(a), int(b)) for a, b in zip(t, o)}

    def cache(self):
        n = self.c.cache_n
        return dict(a=self._arr(self.c.cache_a, n, (n,), np.int32),
                    b=self._arr(self.c.cache_b, n, (n,), np.int32),
                    point=self._arr(self.c.cache_pt, n, (n, 3), 'd'),
                    impulse=self._arr(self.c.cache_imp, n, (n, 3), 'd'))

    def state(self):
        k = self._keep
        return dict(position=k['pos'].copy(), orientation=k['q'].copy(),
                    linear_velocity=k['v'].copy(), angular_velocity=k['w'].copy(),
                    awake=k['awake'].astype(bool), sleep_timer=k['sleep_timer'].copy(),
                    aabb_min=k['aabb_min'][:self.c.n].copy(),
                    aabb_max=k['aabb_max'][:self.c.n].copy(),
                    island=k['island'][:self.c.n].copy())

    def islands(self):
        """Sleep islands of the last step as a set of frozensets of body indices."""
        lab = self._keep['island'][:self.c.n]
        groups = {}
        for i, l in enumerate(lab):
            if l >= 0:
                groups.setdefault(int(l), set()).add(i)
        return {frozenset(g) for g in groups.values()}

    def joint_state(self):
        k = self._keep
        J = self.c.n_joints
        return dict(local_a=k['j_local_a'][:J].copy(), local_b=k['j_local_b'][:J].copy(),
                    length=k['j_length'][:J].copy(), accum=k['j_accum'][:J].copy())

    def set_linear_velocity(self, i, v):
        """Overwrite body ``i``'s linear velocity in place (as a host write to
        ``world.linear_velocity`` between steps does), awake or asleep."""
        self._keep['v'][i] = np.asarray(v, 'd')

    def write_back(self, world):
        """Copy the oracle's body state into ``world``'s columns."""
        n = self.c.n
        k = self._keep
        world._position[:n] = k['pos']; world._orientation[:n] = k['q']
        world._linear_velocity[:n] = k['v']; world._angular_velocity[:n] = k['w']
        world._awake[:n] = k['awake'].astype(bool); world._sleep_timer[:n] = k['sleep_timer']

    def __del__(self):
        try:
            if _LIB is not None:
                _LIB.or_free(C.byref(self.c))
        except Exception:
            pass


_SCALARS = ('n', 'n_shapes', 'n_materials', 'n_pair_friction', 'n_filters', 'n_joints',
            'default_lin_damp', 'default_ang_damp', 'velocity_iterations', 'joint_iterations',
            'sleep_enabled', 'warm_start', 'has_collision', 'restitution_threshold', 'slop',
            'correction', 'margin', 'n_volumes')
_ARRAYS = {name: t for name, t in OrWorldC._fields_ if t in (D, I, U8)}
_OUTPUTS = ('pairs', 'solid', 'c_a', 'c_b', 'c_pt', 'c_n', 'c_depth', 'c_imp', 'cache_a',
            'cache_b', 'cache_pt', 'cache_imp', 'ov_trg', 'ov_other')


def capsule_triangles(p0, p1, radius, verts):
    """``or_capsule_triangles`` with the reference's ``capsule_triangle_batch``
    return convention (collide.py:438-462): ``(hit, points, normals, depths)``,
    zeros where there is no hit."""
    verts = np.ascontiguousarray(verts, dtype='d').reshape(-1, 3, 3)
    n = len(verts)
    hit = np.zeros(n, np.uint8)
    points = np.zeros((n, 3))
    normals = np.zeros((n, 3))
    depths = np.zeros(n)
    a = np.ascontiguousarray(p0, dtype='d')
    b = np.ascontiguousarray(p1, dtype='d')
    if n:
        lib().or_capsule_triangles(_ptr(a, D), _ptr(b, D), float(radius), _ptr(verts, D), n,
                                   _ptr(hit, U8), _ptr(points, D), _ptr(normals, D), _ptr(depths, D))
    return hit.astype(bool), points, normals, depths


def to_arrays(ow):
    """Every oracle input (arrays, scalars, gravity and warm-start cache) as a dict."""
    out = {name: ow._keep[name].copy() for name in _ARRAYS if name in ow._keep}
    for s in _SCALARS:
        out['s_' + s] = np.array(getattr(ow.c, s))
    out['g'] = np.array(list(ow.c.g))
    cache = ow.cache()
    for k, v in cache.items():
        out['cache_' + k] = v
    return out


def from_arrays(d):
    """Rebuild an ``OracleWorld`` from :func:`to_arrays` output."""
    ow = OracleWorld()
    for name, t in _ARRAYS.items():
        if name in d and name not in _OUTPUTS:
            ow._set(name, np.ascontiguousarray(d[name]).copy(), t)
    for s in _SCALARS:
        if 's_' + s in d:
            setattr(ow.c, s, d['s_' + s].item())
    ow.c.g = (C.c_double * 3)(*[float(x) for x in d['g']])
    if len(d['cache_a']):
        ow.set_cache(d['cache_a'], d['cache_b'], d['cache_point'], d['cache_impulse'])
    return ow
