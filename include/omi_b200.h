/*
 * omi_b200 — C ABI of the B200 (sm_100a) rigid-body step.
 *
 * One context owns one CUDA stream and one device-resident "arena": any
 * number of independent worlds, each a contiguous range of body rows in a
 * structure-of-arrays layout identical to the reference's numpy columns
 * (position (n,3), orientation (n,4) xyzw, ...; src/omi_physics/world.py:75-122).
 * A plain PhysicsWorld is an arena of one world; the batched/serving forms
 * step many worlds with the same launches.
 *
 * Conventions: every call returns 0 on success or a negative OMI_E_* code;
 * omi_last_error() gives the message. Host buffers are caller-owned and are
 * never retained past the call. A context is used from one host thread at a
 * time. No call falls back to the CPU: without a usable device they fail.
 */
#ifndef OMI_B200_H
#define OMI_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OMI_OK 0
#define OMI_E_CUDA (-1)         /* CUDA runtime error (message has details) */
#define OMI_E_ARG (-2)          /* bad argument / size */
#define OMI_E_UNSUPPORTED (-3)  /* feature outside the device path (a dynamic triangle mesh ...) */
#define OMI_E_STATE (-4)        /* call out of order (e.g. step before load) */
#define OMI_E_TIMEOUT (-5)      /* a bounded device wait gave up */
#define OMI_E_OOM (-6)          /* arena would exceed the context's HBM budget */
#define OMI_E_LIMIT (-7)        /* the step completed, but some convex pairs outgrew the bounded EPA
                                   polytope and their contacts were dropped (the reference's EPA,
                                   gjk.py:120-217, keeps an unbounded face list) */
#define OMI_E_BOUNDS (-8)       /* bounds-checked build only: a device index check failed; the access
                                   was skipped and the step's results are not valid */

/* Shape types, combine modes, joint types: same meaning as the reference's
 * model.Shape.type, model.combine modes (model.py:231-243) and joints.py. */
/* OMI_SHAPE_CAPSULE also carries the reference's cylinder, which it collides
 * as a capsule (body.py:224-228): shape_radius = radiusBottom,
 * shape_size = (0, height, 0). Capsule pairs go through GJK/EPA. */
enum { OMI_SHAPE_SPHERE = 1, OMI_SHAPE_BOX = 2, OMI_SHAPE_CONVEX = 3, OMI_SHAPE_CAPSULE = 4, OMI_SHAPE_TRIMESH = 5 };
enum { OMI_AVERAGE = 0, OMI_MINIMUM = 1, OMI_MAXIMUM = 2, OMI_MULTIPLY = 3 };
enum { OMI_JOINT_POINT = 0, OMI_JOINT_DISTANCE = 1, OMI_JOINT_MOTOR = 2 };
/* per-world flag bits */
enum { OMI_WF_SLEEP = 1, OMI_WF_WARM = 2, OMI_WF_COLLISION = 4, OMI_WF_ACTIVE = 8 };

/*
 * Scene tables for a whole arena (all worlds concatenated). Body, shape,
 * material and joint indices are global (world-local index + the world's
 * offset); -1 keeps the reference's meaning (no shape / default material /
 * the world as a joint end). Filter rows are world-local: row 0 is the
 * default filter, row f+1 is the world's filters[f]; each world's
 * (rows x rows) collides_with matrix starts at w_filter_off[w].
 * Pair-friction entries are per world, keyed like the reference's
 * PhysicsWorld.pair_friction dict: by the bodies' raw (world-local)
 * collider_material values with a <= b, sorted by (a, b) within each world's
 * range (world.py:207-228); `material_key` carries those raw values per body.
 */
typedef struct OmiScene {
    int32_t n_worlds;
    const int32_t *w_body_off;      /* n_worlds+1 */
    const double *w_gravity;        /* n_worlds*3, resolved (world.py:386-396) */
    const double *w_dt;             /* n_worlds */
    const int32_t *w_iters;         /* velocity iterations */
    const int32_t *w_joint_iters;
    const int32_t *w_flags;         /* OMI_WF_* */
    const double *w_default_damp;   /* n_worlds*2: linear, angular */
    const double *w_solver;         /* n_worlds*2: restitution threshold, slop */
    const int32_t *w_filter_off, *w_filter_rows;
    const int32_t *w_pf_off, *w_pf_n;
    const int32_t *w_joint_off;     /* n_worlds+1 */

    int32_t n_bodies;
    const double *pos, *q, *v, *w;  /* n*3, n*4, n*3, n*3 */
    const double *inv_mass, *inv_inertia;           /* n, n*3 */
    const double *gravity_factor, *lin_damp, *ang_damp, *quad_drag, *sleep_timer;
    const int32_t *motion_type;     /* 0 static, 1 kinematic, 2 dynamic */
    const int32_t *shape;           /* global shape index or -1 */
    const int32_t *material;        /* global material index or -1 (default material) */
    const int32_t *material_key;    /* raw collider_material value (pair-friction key) */
    const int32_t *filter_row;      /* world-local filter row */
    const uint8_t *awake;

    int32_t n_shapes;
    const int32_t *shape_type;
    const double *shape_radius, *shape_size;        /* n_shapes, n_shapes*3 */
    const int32_t *shape_pt_off, *shape_pt_cnt;
    int32_t n_points;
    const double *points;                            /* local convex points */

    int32_t n_materials;
    const double *mat_dynf, *mat_rest;
    const int32_t *mat_fcomb, *mat_rcomb;
    int32_t n_pair_friction;
    const int32_t *pf_a, *pf_b;
    const double *pf_mu;
    int32_t n_filter_bytes;
    const uint8_t *filter_matrix;

    int32_t n_joints;
    const int32_t *j_type, *j_a, *j_b;              /* motor: j_a = body */
    const double *j_anchor, *j_anchor_b, *j_local_a, *j_local_b;   /* *3 */
    const uint8_t *j_has_local_a, *j_has_local_b;
    const double *j_length;
    const uint8_t *j_has_length;
    const double *j_axis, *j_target, *j_max_force, *j_accum;

    /* sensors (triggers.py:17-72): a body's sensor shape (global index) or -1;
     * NULL when no body has one. A pair with a sensor on either body makes no
     * contact; its overlap is tested after the contact solve. */
    const int32_t *trigger_shape;
    /* gravity volumes (gravity.py:51-108), each world's rows in application
     * order (stable by priority); w_vol_off NULL when there are none */
    const int32_t *w_vol_off;       /* n_worlds+1 */
    int32_t n_volumes;
    const int32_t *vol_kind;        /* OMI_VOL_* flags */
    const double *vol_g;            /* field magnitude */
    const double *vol_field;        /* *3: a directional field's acceleration (normalize(direction) *
                                       gravity, as field_at forms it), or a point field's centre */
    const double *vol_rc, *vol_rr;  /* *3: region centre; radius**2 in [0] (sphere) or half-extents (box) */

    /* triangle meshes (body.py:155-212, trigrid.py:63-218): static or kinematic
     * bodies whose collider is an OMI_SHAPE_TRIMESH shape (its points listed as
     * for a hull), each with its triangles in world space and the reference's
     * uniform grid over them, built on the host from the body's pose (and on
     * the device every step for a kinematic mesh, as the reference rebuilds a
     * mesh proxy every step) */
    int32_t n_meshes;
    const int32_t *mesh_body;       /* n_meshes: global body index */
    const int32_t *mesh_tri_off;    /* n_meshes+1: rows of the triangle tables */
    const int32_t *mesh_grid_i;     /* n_meshes*4: exact (fewer than 256 triangles), grid shape (3) */
    const double *mesh_grid_d;      /* n_meshes*7: grid low (3), high (3), cell size */
    const double *tri_verts;        /* n_tris*9: world vertices */
    const double *tri_box;          /* n_tris*6: bounds lo (3), hi (3) */
    const int32_t *tri_cells;       /* n_tris*6: first cell (3), last cell (3) */
    const uint8_t *tri_big;         /* n_tris: spans more than 64 cells (always a candidate) */
    const int32_t *tri_idx;         /* n_tris*3: vertex indices into the mesh shape's points; a kinematic
                                       mesh's tables are rebuilt from them every step */
} OmiScene;

/* gravity volume kind flags: point field (else directional); region sphere,
 * box (else everywhere); replace (overrides) or stop (zeroes), else adds */
enum { OMI_VOL_POINT = 1, OMI_VOL_SPHERE = 2, OMI_VOL_BOX = 4, OMI_VOL_REPLACE = 8, OMI_VOL_STOP = 16 };

typedef struct OmiCtx OmiCtx;

/* ---- context ---------------------------------------------------------- */
int omi_create(int device, OmiCtx **out);
int omi_destroy(OmiCtx *ctx);
const char *omi_last_error(OmiCtx *ctx);
/* Launch on this cudaStream_t (NULL = the context's own stream). */
int omi_set_stream(OmiCtx *ctx, void *stream);
/* Refuse arenas whose device footprint exceeds this many bytes (0 = none). */
int omi_set_budget(OmiCtx *ctx, int64_t bytes);
int64_t omi_device_bytes(OmiCtx *ctx);
/* Lower the device's safety bounds, for tests and diagnostics (no counterpart
 * in the reference, whose sweep never waits and whose EPA is unbounded):
 * spin_limit = polls before a contact-sweep wait gives up (the step then
 * fails with OMI_E_TIMEOUT), epa_faces = EPA polytope faces (4..512; a pair
 * past it is dropped and the step reports OMI_E_LIMIT), stall_run = a
 * world-local run index whose sweep entries are made to wait forever in
 * every world (-1 = none), so a test can make a wait run out. 0 restores a
 * default. Applies to the next step (the step graph is re-captured). */
int omi_set_limits(OmiCtx *ctx, int32_t spin_limit, int32_t epa_faces, int32_t stall_run);
/* 1 in the bounds-checked debug build of this library (_omi_b200_checked.so,
 * compiled with -DOMI_BOUNDS_CHECK), else 0. No counterpart in the reference
 * (its Cython accelerators are compiled with boundscheck=False). The checked
 * build tests the indices the step's kernels take from data (pair and contact
 * bodies, shapes and hull point ranges, filter rows, solver-row bodies,
 * sweep successors, joint bodies) before using them; a failed check skips
 * the access, is counted on the device, and omi_step / omi_sync return
 * OMI_E_BOUNDS naming the first one. Nothing traps. The shipped build
 * compiles the checks out. */
int omi_bounds_checked(void);
/* Test hook of the bounds-checked build: from the next step on, the
 * narrowphase checks candidate pair `pair` (its index in omi_get_pairs'
 * list) as if its first body index were past the arena, so the check fails
 * and the step returns OMI_E_BOUNDS; -1 turns it off. One setting per
 * device, shared by every context on it. The shipped build returns
 * OMI_E_UNSUPPORTED. No counterpart in the reference. */
int omi_bounds_probe(OmiCtx *ctx, int32_t pair);
/* Launch configuration of the step's kernels (no counterpart in the
 * reference): results do not depend on it, only speed, so an autotuner may
 * pick it per GPU and workload. sweep_warps = warps per contact-sweep block
 * (4 or 8), sweep_max_split = sweep groups a block may split into once its
 * worlds are small (1, 2, 4), pair_block / pair_blocks_per_sm = block size
 * (128/256/512) and blocks per SM (1-32) of the pair count and emit passes,
 * narrow_block = block size of the analytic narrowphase and clipping (64,
 * 128, 256), gjk_warps = warps (one pair each) per GJK/EPA block (2, 4, 8).
 * Defaults: 8, 4, 256, 16, 128, 4, 16, 16 (8 on a GPU without 16-CTA clusters), 32.
 * A change re-captures the step graph. */
typedef struct OmiTuning {
    int32_t sweep_warps, sweep_max_split, pair_block, pair_blocks_per_sm, narrow_block, gjk_warps;
    /* blocks of a wide world's contact sweep (1-148; 1 = the one-block sweep with its
     * shared-memory staging, the others share the work through device memory) */
    int32_t wide_sweep_blocks;
    /* 8 or 16: a wide world's contact sweep on one thread-block cluster of that many CTAs
     * (each owning a slab of the runs, crossing entries through distributed shared
     * memory) while every CTA's body records fit its shared memory, else on
     * wide_sweep_blocks blocks (the cluster sweeps every world when that is 1); 0 = off */
    int32_t wide_cluster;
    /* ready contact-sweep entries a warp claims at once (8, 16 or 32): fewer leave more
     * warps free to take an entry the moment it becomes ready */
    int32_t sweep_claim;
} OmiTuning;
int omi_set_tuning(OmiCtx *ctx, const OmiTuning *tuning);
int omi_get_tuning(OmiCtx *ctx, OmiTuning *tuning);
/* Colliding worlds with more bodies than this are "wide": their sort, sweep
 * links, wake, contact sweep, warm-start cache store, positions and sleep
 * run on many blocks instead of one block per world (the same results, bit
 * for bit). Default 3072; 0 makes every colliding world wide. Applies from
 * the next omi_load / omi_reserve_slots. (No counterpart in the reference.) */
int omi_set_wide_threshold(OmiCtx *ctx, int32_t bodies);
/* Shared-memory ints each CTA of the wide contact sweep's thread-block
 * cluster may use (0, the default: all it has). The cluster sweeps a wide
 * world whose body records fit its CTAs' shared memory and hands any other
 * to the many-block sweep (unless wide_sweep_blocks is 1); a smaller budget
 * makes it hand off smaller worlds - the same results, bit for bit. (No
 * counterpart in the reference.) */
int omi_set_cluster_budget(OmiCtx *ctx, int32_t ints);
/* Check a scene the way omi_load does, on the host only (no device, no
 * context): every index a kernel would follow is range-checked. Returns 0 or
 * the status omi_load would return, with the message in err (err_cap bytes,
 * may be NULL). omi_load refuses a scene that fails this check and keeps the
 * arena it had loaded before. */
int omi_validate_scene(const OmiScene *scene, char *err, int32_t err_cap);

/* ---- scene ------------------------------------------------------------ */
/* Upload a whole arena (replaces any previous one). Builds what the reference
 * builds lazily on the first step: _build_refit_cache (world.py:443-469). */
int omi_load(OmiCtx *ctx, const OmiScene *scene);
/* Which worlds take part in the next steps (n_worlds bytes, 0/1). */
int omi_set_active(OmiCtx *ctx, const uint8_t *active);
/* Per-world step parameters (any pointer may be NULL to keep the current
 * values): dt, velocity iterations, joint iterations, OMI_WF_* flags. */
int omi_set_world_params(OmiCtx *ctx, const double *dt, const int32_t *iters,
                         const int32_t *joint_iters, const int32_t *flags);

/* ---- serving slots ------------------------------------------------------ */
/* Capacities of one slot: an arena of n_slots empty, inactive worlds, each
 * able to hold one world within these limits. */
typedef struct OmiSlotCaps {
    int32_t bodies, shapes, materials, points, joints, filter_rows, pair_friction;
} OmiSlotCaps;
int omi_reserve_slots(OmiCtx *ctx, int32_t n_slots, const OmiSlotCaps *caps);
/* The same with capacities per slot (caps[n_slots]): slots of several size
 * classes in one arena, so small requests do not hold large slots. */
int omi_reserve_slots_each(OmiCtx *ctx, int32_t n_slots, const OmiSlotCaps *caps);
/* Admit one world (an OmiScene with n_worlds == 1, local indices) into a
 * slot: its tables and state are copied in, its warm-start cache cleared and
 * the slot activated when OMI_WF_ACTIVE is set. No reallocation, no graph
 * rebuild: other slots keep stepping in the same launches. */
int omi_load_world(OmiCtx *ctx, int32_t slot, const OmiScene *one);
/* First arena row of a world and its live body count. */
int omi_world_rows(OmiCtx *ctx, int32_t world, int32_t *first_row, int32_t *n_bodies);

/* ---- state transfer (host columns <-> device arena) ------------------- */
/* Rows [begin, begin+count) of the arena; any pointer may be NULL to skip. */
int omi_upload_state(OmiCtx *ctx, int32_t begin, int32_t count, const double *pos,
                     const double *q, const double *v, const double *w,
                     const uint8_t *awake, const double *sleep_timer);
int omi_download_state(OmiCtx *ctx, int32_t begin, int32_t count, double *pos, double *q,
                       double *v, double *w, uint8_t *awake, double *sleep_timer,
                       double *aabb_min, double *aabb_max);
/* Joint state the reference keeps on the constraint objects
 * (joints.py:88-91 local anchors, 151-152 rest length, 201 motor accum). */
int omi_download_joints(OmiCtx *ctx, double *local_a, double *local_b, uint8_t *has_local_a,
                        uint8_t *has_local_b, double *length, uint8_t *has_length,
                        double *accum);

/* Warm-start cache of one world, the reference's SequentialImpulseSolver._cache
 * (solver.py:91, 272-278) flattened in insertion order: entry i is the pair
 * (a[i], b[i]) (global body indices), its contact point (3) and accumulated
 * impulses (normal, tangent0, tangent1). set replaces it; get returns the
 * entry count (or a negative status), writing at most cap entries. */
int omi_set_cache(OmiCtx *ctx, int32_t world, int32_t n, const int32_t *a, const int32_t *b,
                  const double *point, const double *impulse);
int omi_get_cache(OmiCtx *ctx, int32_t world, int32_t *a, int32_t *b, double *point,
                  double *impulse, int32_t cap);

/* ---- the step --------------------------------------------------------- */
/* n_steps x PhysicsWorld.step(dt) (world.py:410-430) for every active world,
 * each world with its own dt: integrate forces, refit, broadphase,
 * narrowphase, contact solve, joints, integrate positions, sleep. Captured as
 * a CUDA graph after the first step; capacity overflow is detected before any
 * state changes, regrown and the step re-run, so results do not depend on it. */
int omi_step(OmiCtx *ctx, int32_t n_steps);
/* Same, enqueued without the final host synchronisation (use omi_sync). */
int omi_step_async(OmiCtx *ctx, int32_t n_steps);
int omi_sync(OmiCtx *ctx);

/* ---- stage entry points (the backend seam and the collision stages) ---- */
/* NumpyBackend.integrate_forces (backend.py:26-40) */
int omi_integrate_forces(OmiCtx *ctx);
/* NumpyBackend.refit_aabbs -> PhysicsWorld.refit_aabbs (backend.py:51-53, world.py:471-508) */
int omi_refit_aabbs(OmiCtx *ctx);
/* BroadPhase.pairs (broadphase.py:243-294): pair lists per world, in the
 * reference's order; returns OMI_E_ARG-free status, counts via omi_counts */
int omi_broadphase(OmiCtx *ctx);
/* solid-pair filter + NarrowPhase.generate (world.py:661-671, narrowphase.py:51-100,
 * _collide_native.box_box/sphere_sphere/sphere_box, gjk.collide_convex) */
int omi_narrowphase(OmiCtx *ctx);
/* SequentialImpulseSolver.solve (solver.py:192-278 -> _solver_native.prepare_and_solve,
 * _solver_native.pyx:179-312), warm-start cache kept on the device */
int omi_solve_contacts(OmiCtx *ctx);
/* PhysicsWorld._solve_joints (world.py:599-611, joints.py:60-212) */
int omi_solve_joints(OmiCtx *ctx);
/* NumpyBackend.integrate_positions (backend.py:42-49) */
int omi_integrate_positions(OmiCtx *ctx);
/* PhysicsWorld._update_sleep (world.py:510-567) */
int omi_update_sleep(OmiCtx *ctx);

/* ---- results of the last step ----------------------------------------- */
/* per-world pair and contact counts (n_worlds each) */
int omi_counts(OmiCtx *ctx, int32_t *pairs, int32_t *contacts);
/* broadphase pairs of one world as global body indices (2*cap int32) */
int omi_get_pairs(OmiCtx *ctx, int32_t world, int32_t *out, int32_t cap);
/* contacts of one world (Contact records, collide.py:37-53) with the solver's
 * accumulated impulses (normal, tangent0, tangent1); the impulses are zero when
 * the world's warm start is off, as the reference leaves its contacts then
 * (solver.py:271-278) */
int omi_get_contacts(OmiCtx *ctx, int32_t world, int32_t *a, int32_t *b, double *point,
                     double *normal, double *depth, double *impulse, int32_t cap);
/* sleep-island label per body of one world (-1 = not in contact) */
int omi_get_islands(OmiCtx *ctx, int32_t world, int32_t *labels);

/* This step's sensor overlaps in `world` (TriggerSystem.overlaps after
 * triggers.update, triggers.py:24-44): (trigger body, other body) pairs with
 * world-local indices, sorted, at most `cap` written. Returns the count (which
 * may exceed cap) or a negative OMI_E_*. Enter / stay / exit events are the
 * difference between consecutive steps' sets, formed by the caller. */
int omi_get_trigger_overlaps(OmiCtx *ctx, int32_t world, int32_t *trg, int32_t *other, int32_t cap);

/* ---- capsule against triangles (the character controller's query) ----
 *
 * The compiled capsule_triangles (_collide_native.pyx:454-574), reached from
 * collide.capsule_triangle_batch / capsule_triangles / capsule_mesh_pushes
 * (collide.py:385-462) and the mesh route of collide.collide
 * (collide.py:272-306). A capsule is the segment p0-p1 with a radius; verts
 * is (n, 3, 3) (triangle, vertex, axis). For every triangle: hit (1 byte),
 * point on the triangle (3), normal from the triangle toward the capsule (3)
 * and depth, bit-identical to the reference's; triangles without contact get
 * hit 0 and zeros, as the arrays capsule_triangle_batch passes in hold.
 * These calls need no loaded scene. */

/* One capsule, host buffers: the reference's
 * _native.capsule_triangles(cp0, cp1, radius, verts, hit, points, normals,
 * depths) (_collide_native.pyx:454-574). Returns when the outputs are written. */
int omi_capsule_triangles(OmiCtx *ctx, const double *p0, const double *p1, double radius,
                          const double *verts, int64_t n, uint8_t *hit, double *points,
                          double *normals, double *depths);
/* q capsules at once, host buffers: caps is (q, 7) = p0 (3), p1 (3), radius;
 * the triangles of capsule c are rows [tri_off[c], tri_off[c+1]) of verts,
 * with tri_off[0] = 0, tri_off[q] = n and non-decreasing (checked). Copies in,
 * computes and copies out in chunks on two internal streams, so transfers
 * overlap the kernel (pinned host buffers let them run asynchronously).
 * Returns when the outputs are written. */
int omi_capsule_triangles_batch(OmiCtx *ctx, int32_t q, const double *caps, const int64_t *tri_off,
                                const double *verts, int64_t n, uint8_t *hit, double *points,
                                double *normals, double *depths);
/* The same on DEVICE buffers, enqueued on the context's stream (omi_set_stream);
 * returns without waiting. tri_off is not checked here: a malformed one gives
 * wrong answers but every read stays inside caps (q rows) and tri_off (q+1). */
int omi_capsule_triangles_device(OmiCtx *ctx, int32_t q, const double *caps, const int64_t *tri_off,
                                 const double *verts, int64_t n, uint8_t *hit, double *points,
                                 double *normals, double *depths);
/*
 * Allocation-free sweep-and-prune for one world. (This entry point has no
 * counterpart in the reference.) It is for callers that must not allocate
 * device memory: an engine whose memory is fully reserved up front by its own
 * pool, a real-time loop where cudaMalloc/cudaFree would synchronise the
 * device mid-frame, or code running where the allocator is unavailable.
 * Contract: bodies are sorted by aabb_min.x (stable: ties by index, NaN
 * last); for each body in that order, every later body whose min.x is at
 * most its max.x and whose y and z ranges overlap (>=) forms a pair, kept
 * when at least one of the two is dynamic (motion_type 2) and the filter
 * matrix lets their rows collide. Pairs are written as (min, max) body
 * indices, ordered by the first body's sorted position, then the second's.
 * This is the same list, in the same order, as omi_broadphase gives.
 *
 * All array arguments are DEVICE pointers owned by the caller: aabb_min and
 * aabb_max (n*3 doubles), motion_type (n ints), optionally filter_row (n ints,
 * rows of the filter_rows x filter_rows collides_with matrix filter_matrix,
 * each entry in [0, filter_rows): the kernel does not check them; both NULL
 * when every pair collides), the output pairs (2*pair_cap ints,
 * (min, max) body indices) and n_pairs (1 int: the full pair count, which may
 * exceed pair_cap; pairs past pair_cap are not written). Work is enqueued on
 * `stream` (a cudaStream_t, NULL = default) and the call returns without
 * waiting; read n_pairs after the stream is synchronised.
 *
 * Scratch lives in a fixed device array inside this library (about 0.8 MB,
 * held by every GPU that loads the library until the process exits), so
 * n_bodies may not exceed OMI_NOALLOC_MAX_BODIES: larger worlds are refused
 * with OMI_E_ARG and a message in err (err_cap bytes, may be NULL). The first
 * call on each device looks that array's device address up (once per device,
 * with the device current, serialised between host threads); make that first
 * call before any stream capture, and do not call it on a device after a
 * cudaDeviceReset there (the looked-up address belonged to the old context).
 * Every call shares the one array, so calls whose work overlaps on the GPU
 * (other streams, other host threads) race and must be serialised by the
 * caller. No call allocates or frees memory.
 */
#define OMI_NOALLOC_MAX_BODIES 16384
int omi_sweep_pairs_noalloc(const double *aabb_min, const double *aabb_max,
                            const int32_t *motion_type, const int32_t *filter_row,
                            const uint8_t *filter_matrix, int32_t filter_rows, int32_t n_bodies,
                            int32_t *pairs, int32_t pair_cap, int32_t *n_pairs, void *stream,
                            char *err, int32_t err_cap);

/* Critical path of each world's last contact sweep (n_worlds ints;
 * diagnostics): the longest chain of runs that must follow one another,
 * weighted by their contact counts - the sequential sweep's length in contact
 * solves, after independent runs are overlapped. A wide world's sweep does
 * not track it: -1 when a thread-block cluster swept it, -2 when the
 * many-block sweep did. No counterpart in the reference (whose sweep is the
 * full sequence). */
int omi_world_levels(OmiCtx *ctx, int32_t *levels);

/* per-kernel device time (ms) of the last profiled step, see omi_profile_step */
int omi_profile_step(OmiCtx *ctx, float *ms, int32_t n, int32_t *n_out);
const char *omi_kernel_name(int32_t i);
/* launches of the library's own kernels since load */
int64_t omi_launch_count(OmiCtx *ctx);

#ifdef __cplusplus
}
#endif
#endif
