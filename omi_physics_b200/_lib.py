"""ctypes binding of the CUDA library ``_omi_b200.so`` (include/omi_b200.h).

The library is built in-tree (``python -m omi_physics_b200.build`` or
``__graft_entry__.build()``); importing this module does not build it, and
every entry point fails loudly when it is missing or no CUDA device is
usable — there is no CPU fallback anywhere in the package.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
#: the shipped library, and its bounds-checked debug build (device index
#: checks that report OMI_E_BOUNDS instead of reading out of range), which
#: ``OMI_B200_CHECKED=1`` in the environment selects for the whole process
LIB_PATH_SHIPPED = os.path.join(HERE, '_omi_b200.so')
LIB_PATH_CHECKED = os.path.join(HERE, '_omi_b200_checked.so')
LIB_PATH = LIB_PATH_CHECKED if os.environ.get('OMI_B200_CHECKED', '') not in ('', '0') else LIB_PATH_SHIPPED

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int32)
I64 = C.POINTER(C.c_int64)
U8 = C.POINTER(C.c_uint8)

OMI_E_CUDA, OMI_E_ARG, OMI_E_UNSUPPORTED, OMI_E_STATE, OMI_E_TIMEOUT, OMI_E_OOM, OMI_E_LIMIT, OMI_E_BOUNDS = (
    -1, -2, -3, -4, -5, -6, -7, -8)
WF_SLEEP, WF_WARM, WF_COLLISION, WF_ACTIVE = 1, 2, 4, 8


class OmiError(RuntimeError):
    """A failed library call; ``code`` is the negative OMI_E_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__('%s (status %d)' % (msg, code))
        self.code = code


class UnsupportedFeature(OmiError):
    """The scene uses something outside the device path (triggers, trimesh ...)."""


class OutOfBudget(OmiError):
    """The arena would exceed the context's device-memory budget."""


class SweepTimeout(OmiError):
    """A bounded wait of the contact sweep ran out: the step did not complete
    (the worlds' state is partly advanced; restore it before stepping on)."""


class EpaLimit(OmiError):
    """The step completed, but some convex pairs outgrew the bounded EPA
    polytope and their contacts were dropped (the reference's EPA is unbounded)."""


class BoundsError(OmiError):
    """Bounds-checked build only: a device index check failed (the access was
    skipped, the step's results are not valid); the message names the first."""


class OmiScene(C.Structure):
    """Mirror of ``struct OmiScene``."""
    _fields_ = [
        ('n_worlds', C.c_int32),
        ('w_body_off', I), ('w_gravity', D), ('w_dt', D), ('w_iters', I), ('w_joint_iters', I),
        ('w_flags', I), ('w_default_damp', D), ('w_solver', D),
        ('w_filter_off', I), ('w_filter_rows', I), ('w_pf_off', I), ('w_pf_n', I),
        ('w_joint_off', I),
        ('n_bodies', C.c_int32),
        ('pos', D), ('q', D), ('v', D), ('w', D), ('inv_mass', D), ('inv_inertia', D),
        ('gravity_factor', D), ('lin_damp', D), ('ang_damp', D), ('quad_drag', D),
        ('sleep_timer', D),
        ('motion_type', I), ('shape', I), ('material', I), ('material_key', I),
        ('filter_row', I), ('awake', U8),
        ('n_shapes', C.c_int32), ('shape_type', I), ('shape_radius', D), ('shape_size', D),
        ('shape_pt_off', I), ('shape_pt_cnt', I), ('n_points', C.c_int32), ('points', D),
        ('n_materials', C.c_int32), ('mat_dynf', D), ('mat_rest', D), ('mat_fcomb', I),
        ('mat_rcomb', I),
        ('n_pair_friction', C.c_int32), ('pf_a', I), ('pf_b', I), ('pf_mu', D),
        ('n_filter_bytes', C.c_int32), ('filter_matrix', U8),
        ('n_joints', C.c_int32), ('j_type', I), ('j_a', I), ('j_b', I),
        ('j_anchor', D), ('j_anchor_b', D), ('j_local_a', D), ('j_local_b', D),
        ('j_has_local_a', U8), ('j_has_local_b', U8), ('j_length', D), ('j_has_length', U8),
        ('j_axis', D), ('j_target', D), ('j_max_force', D), ('j_accum', D),
        ('trigger_shape', I),
        ('w_vol_off', I), ('n_volumes', C.c_int32), ('vol_kind', I), ('vol_g', D), ('vol_field', D),
        ('vol_rc', D), ('vol_rr', D),
        ('n_meshes', C.c_int32), ('mesh_body', I), ('mesh_tri_off', I), ('mesh_grid_i', I),
        ('mesh_grid_d', D), ('tri_verts', D), ('tri_box', D), ('tri_cells', I), ('tri_big', U8),
        ('tri_idx', I),
    ]


class OmiSlotCaps(C.Structure):
    """Mirror of ``struct OmiSlotCaps``."""
    _fields_ = [(n, C.c_int32) for n in ('bodies', 'shapes', 'materials', 'points', 'joints',
                                          'filter_rows', 'pair_friction')]


class OmiTuning(C.Structure):
    """Mirror of ``struct OmiTuning`` (the step's launch configuration)."""
    _fields_ = [(n, C.c_int32) for n in ('sweep_warps', 'sweep_max_split', 'pair_block',
                                          'pair_blocks_per_sm', 'narrow_block', 'gjk_warps',
                                          'wide_sweep_blocks', 'wide_cluster', 'sweep_claim')]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


#: the library's default launch configuration
DEFAULT_TUNING = dict(sweep_warps=8, sweep_max_split=4, pair_block=256, pair_blocks_per_sm=16,
                      narrow_block=128, gjk_warps=4, wide_sweep_blocks=16, wide_cluster=16,
                      sweep_claim=32)

#: every symbol include/omi_b200.h declares, with (restype, argtypes)
PROTOTYPES = {
    'omi_create': (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    'omi_destroy': (C.c_int, [C.c_void_p]),
    'omi_last_error': (C.c_char_p, [C.c_void_p]),
    'omi_set_stream': (C.c_int, [C.c_void_p, C.c_void_p]),
    'omi_set_budget': (C.c_int, [C.c_void_p, C.c_int64]),
    'omi_device_bytes': (C.c_int64, [C.c_void_p]),
    'omi_set_limits': (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    'omi_bounds_checked': (C.c_int, []),
    'omi_bounds_probe': (C.c_int, [C.c_void_p, C.c_int32]),
    'omi_validate_scene': (C.c_int, [C.POINTER(OmiScene), C.c_char_p, C.c_int32]),
    'omi_set_tuning': (C.c_int, [C.c_void_p, C.POINTER(OmiTuning)]),
    'omi_get_tuning': (C.c_int, [C.c_void_p, C.POINTER(OmiTuning)]),
    'omi_set_wide_threshold': (C.c_int, [C.c_void_p, C.c_int32]),
    'omi_set_cluster_budget': (C.c_int, [C.c_void_p, C.c_int32]),
    'omi_load': (C.c_int, [C.c_void_p, C.POINTER(OmiScene)]),
    'omi_set_active': (C.c_int, [C.c_void_p, U8]),
    'omi_set_world_params': (C.c_int, [C.c_void_p, D, I, I, I]),
    'omi_reserve_slots': (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(OmiSlotCaps)]),
    'omi_reserve_slots_each': (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(OmiSlotCaps)]),
    'omi_load_world': (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(OmiScene)]),
    'omi_world_rows': (C.c_int, [C.c_void_p, C.c_int32, I, I]),
    'omi_upload_state': (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, D, D, D, D, U8, D]),
    'omi_download_state': (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, D, D, D, D, U8, D, D, D]),
    'omi_download_joints': (C.c_int, [C.c_void_p, D, D, U8, U8, D, U8, D]),
    'omi_set_cache': (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, I, I, D, D]),
    'omi_get_cache': (C.c_int, [C.c_void_p, C.c_int32, I, I, D, D, C.c_int32]),
    'omi_step': (C.c_int, [C.c_void_p, C.c_int32]),
    'omi_step_async': (C.c_int, [C.c_void_p, C.c_int32]),
    'omi_sync': (C.c_int, [C.c_void_p]),
    'omi_integrate_forces': (C.c_int, [C.c_void_p]),
    'omi_refit_aabbs': (C.c_int, [C.c_void_p]),
    'omi_broadphase': (C.c_int, [C.c_void_p]),
    'omi_narrowphase': (C.c_int, [C.c_void_p]),
    'omi_solve_contacts': (C.c_int, [C.c_void_p]),
    'omi_solve_joints': (C.c_int, [C.c_void_p]),
    'omi_integrate_positions': (C.c_int, [C.c_void_p]),
    'omi_update_sleep': (C.c_int, [C.c_void_p]),
    'omi_counts': (C.c_int, [C.c_void_p, I, I]),
    'omi_get_pairs': (C.c_int, [C.c_void_p, C.c_int32, I, C.c_int32]),
    'omi_get_contacts': (C.c_int, [C.c_void_p, C.c_int32, I, I, D, D, D, D, C.c_int32]),
    'omi_get_islands': (C.c_int, [C.c_void_p, C.c_int32, I]),
    'omi_world_levels': (C.c_int, [C.c_void_p, I]),
    'omi_profile_step': (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int32, I]),
    'omi_kernel_name': (C.c_char_p, [C.c_int32]),
    'omi_launch_count': (C.c_int64, [C.c_void_p]),
    'omi_get_trigger_overlaps': (C.c_int, [C.c_void_p, C.c_int32, I, I, C.c_int32]),
    'omi_capsule_triangles': (C.c_int, [C.c_void_p, D, D, C.c_double, D, C.c_int64, U8, D, D, D]),
    'omi_capsule_triangles_batch': (C.c_int, [C.c_void_p, C.c_int32, D, I64, D,
                                              C.c_int64, U8, D, D, D]),
    'omi_capsule_triangles_device': (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p]),
    'omi_sweep_pairs_noalloc': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                          C.c_int32, C.c_void_p, C.c_void_p, C.c_char_p,
                                          C.c_int32]),
}

#: the fixed body limit of omi_sweep_pairs_noalloc (OMI_NOALLOC_MAX_BODIES)
NOALLOC_MAX_BODIES = 16384

_LIB = None


def load_library():
    """Load ``_omi_b200.so`` (raising if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise OmiError(OMI_E_STATE, 'CUDA library %s is not built; run `python -m omi_physics_b200.build%s`'
                           % (LIB_PATH, ' --checked' if LIB_PATH == LIB_PATH_CHECKED else ''))
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def validate_scene(scene) -> None:
    """Check an :class:`OmiScene` as ``omi_load`` does, on the host only (no
    device needed); raise the matching :class:`OmiError` if it is refused."""
    lib = load_library()
    err = C.create_string_buffer(512)
    rc = lib.omi_validate_scene(C.byref(scene), err, len(err))
    if rc < 0:
        cls = {OMI_E_UNSUPPORTED: UnsupportedFeature}.get(rc, OmiError)
        raise cls(rc, 'omi_validate_scene: ' + err.value.decode())


def ptr(a, t):
    """ctypes pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(t)


class Context:
    """One library context: a CUDA stream and a device arena.

    ``OMI_WIDE_THRESHOLD`` in the environment sets the body count above which
    a world's per-world stages run on many blocks (``omi_set_wide_threshold``)
    for every new context."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.omi_create(int(device), C.byref(h))
        self.h = h
        if rc != 0:
            msg = self.lib.omi_last_error(h).decode() if h.value else 'omi_create failed'
            if h.value:
                self.lib.omi_destroy(h)
                self.h = C.c_void_p()
            raise OmiError(rc, msg)
        self._keep = []
        wide = os.environ.get('OMI_WIDE_THRESHOLD')
        if wide:
            self.call('set_wide_threshold', int(wide))

    def check(self, rc: int, what: str = '') -> int:
        """Raise the matching exception for a negative status; return rc."""
        if rc < 0:
            msg = self.lib.omi_last_error(self.h).decode() or what
            cls = {OMI_E_UNSUPPORTED: UnsupportedFeature, OMI_E_OOM: OutOfBudget, OMI_E_TIMEOUT: SweepTimeout,
                   OMI_E_LIMIT: EpaLimit, OMI_E_BOUNDS: BoundsError}.get(rc, OmiError)
            raise cls(rc, '%s: %s' % (what, msg) if what else msg)
        return rc

    def call(self, name: str, *args) -> int:
        return self.check(getattr(self.lib, 'omi_' + name)(self.h, *args), 'omi_' + name)

    def close(self):
        if getattr(self, 'h', None) is not None and self.h.value:
            self.lib.omi_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- convenience ------------------------------------------------------
    def launches(self) -> int:
        return int(self.lib.omi_launch_count(self.h))

    def device_bytes(self) -> int:
        return int(self.lib.omi_device_bytes(self.h))

    def set_limits(self, spin_limit: int = 0, epa_faces: int = 0, stall_run: int = -1) -> None:
        """Lower the sweep's wait bound or the EPA face bound, or stall one run
        (tests of the failure paths); zeros restore the defaults."""
        self.call('set_limits', int(spin_limit), int(epa_faces), int(stall_run))

    def set_tuning(self, **cfg) -> None:
        """Set the launch configuration (keys of :data:`DEFAULT_TUNING`; missing
        keys keep their current values)."""
        cur = self.tuning()
        cur.update(cfg)
        t = OmiTuning(**{k: int(cur[k]) for k in DEFAULT_TUNING})
        self.call('set_tuning', C.byref(t))

    def set_cluster_budget(self, ints: int = 0) -> None:
        """Shared-memory ints per CTA of the wide sweep's cluster (0: all);
        smaller budgets hand smaller wide worlds to the many-block sweep."""
        self.call('set_cluster_budget', int(ints))

    def tuning(self) -> dict:
        t = OmiTuning()
        self.call('get_tuning', C.byref(t))
        return t.as_dict()

    def profile_step(self):
        """Per-kernel-group device time (ms) of one eagerly launched step."""
        buf = (C.c_float * 32)()
        n = C.c_int32()
        self.call('profile_step', buf, 32, C.byref(n))
        return {self.lib.omi_kernel_name(i).decode(): float(buf[i]) for i in range(n.value)}
