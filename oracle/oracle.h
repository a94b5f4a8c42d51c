/*
 * Oracle (test infrastructure only): a sequential CPU restatement of
 * omi_physics' PhysicsWorld.step (reference v0.3.1) in plain C, float64.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library, and only as the parity reference or the CPU baseline. The
 * product (omi_physics_b200) never links or calls it.
 *
 * Parity pin: tests/golden/ holds fixtures produced by running the reference
 * itself (built from its own sources by oracle/build_ref.sh) and
 * tests/test_oracle_golden.py checks this oracle against them.
 *
 * All arrays are caller-owned, row-major, numpy-compatible. The oracle owns
 * only the per-step outputs (pairs, contacts, islands) and the warm-start
 * cache, which it allocates and frees itself.
 */
#ifndef OMI_ORACLE_H
#define OMI_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* shape types */
/* capsule also stands for the reference's cylinder, which it collides as a
 * capsule (body.py:224-228); shape_radius = radiusBottom, shape_size[1] = height */
enum { OR_SHAPE_SPHERE = 1, OR_SHAPE_BOX = 2, OR_SHAPE_CONVEX = 3, OR_SHAPE_CAPSULE = 4, OR_SHAPE_TRIMESH = 5 };
/* combine modes (model.py:231-243) */
enum { OR_AVERAGE = 0, OR_MINIMUM = 1, OR_MAXIMUM = 2, OR_MULTIPLY = 3 };
/* joint types (joints.py) */
enum { OR_JOINT_POINT = 0, OR_JOINT_DISTANCE = 1, OR_JOINT_MOTOR = 2 };

typedef struct OrWorld {
    /* ---- bodies (world.py:75-122), n rows each ---- */
    int32_t n;
    double *pos, *q, *v, *w, *prev_pos, *prev_q;       /* n*3, n*4 */
    double *inv_mass, *inv_inertia;                      /* n, n*3 */
    double *gravity_factor, *lin_damp, *ang_damp, *quad_drag, *sleep_timer;
    int32_t *motion_type, *collider_shape, *collider_material, *collider_filter;
    uint8_t *awake;
    double *aabb_min, *aabb_max;                         /* n*3 (output of refit) */
    /* ---- shapes ---- */
    int32_t n_shapes;
    int32_t *shape_type;                                 /* OR_SHAPE_* */
    double *shape_radius, *shape_size;                   /* n_shapes, n_shapes*3 */
    int32_t *shape_pt_off, *shape_pt_cnt;                /* convex point ranges */
    double *points;                                      /* local convex points, *3 */
    /* ---- materials (model.py:121-127) ---- */
    int32_t n_materials;
    double *mat_dynf, *mat_rest;
    int32_t *mat_fcomb, *mat_rcomb;
    int32_t n_pair_friction;                             /* world.py:207-228 */
    int32_t *pf_a, *pf_b;                                /* a <= b */
    double *pf_mu;                                       /* dynamic mu */
    /* ---- collision filters: (n_filters+1)^2 matrix, row/col 0 = default ---- */
    int32_t n_filters;
    uint8_t *filter_matrix;
    /* ---- joints (joints.py:60-212), registration order ---- */
    int32_t n_joints;
    int32_t *j_type, *j_a, *j_b;                         /* motor: j_a = body */
    double *j_anchor, *j_anchor_b;                       /* *3 */
    double *j_local_a, *j_local_b;                       /* *3, lazily set */
    uint8_t *j_has_local_a, *j_has_local_b;
    double *j_length; uint8_t *j_has_length;
    double *j_axis, *j_target, *j_max_force, *j_accum;
    /* ---- parameters ---- */
    double g[3];                 /* resolved gravity vector (world.py:386-396) */
    double dt;
    double default_lin_damp, default_ang_damp;
    int32_t velocity_iterations, joint_iterations;
    int32_t sleep_enabled, warm_start, has_collision;
    double restitution_threshold, slop, correction, margin;
    /* ---- warm-start cache (solver.py:91, 272-278), oracle-owned ---- */
    int32_t cache_n;
    int32_t *cache_a, *cache_b;
    double *cache_pt, *cache_imp;                        /* *3, *3 (n, t0, t1) */
    /* ---- per-step outputs, oracle-owned ---- */
    int32_t n_pairs, n_solid;
    int32_t *pairs, *solid;                              /* *2 */
    int32_t n_contacts;
    int32_t *c_a, *c_b;
    double *c_pt, *c_n, *c_depth, *c_imp;                /* *3, *3, 1, *3 */
    int32_t *island;                                     /* n: sleep-island label or -1 */
    /* ---- triggers (triggers.py:17-72): sensor shape per body, -1 none;
     *      NULL means no body has one ---- */
    int32_t *trigger_shape;
    /* ---- gravity volumes (gravity.py:51-108), in application order (stable
     *      by priority): kind = OR_VOL_* flags, g = field magnitude, field =
     *      directional acceleration or point centre (*3), rc = region centre
     *      (*3), rr = sphere radius**2 in [0] or box half-extents (*3) ---- */
    int32_t n_volumes;
    int32_t *vol_kind;
    double *vol_g, *vol_field, *vol_rc, *vol_rr;
    /* ---- per-step trigger overlaps (trigger, other) in pair order, oracle-owned ---- */
    int32_t n_overlaps;
    int32_t *ov_trg, *ov_other;
    /* ---- triangle meshes (body.py:155-212): a trimesh shape's triangles are
     *      rows [shape_tri_off, +shape_tri_cnt) of tris, vertex indices into
     *      the shape's own points (shape_pt_off / shape_pt_cnt) ---- */
    int32_t *shape_tri_off, *shape_tri_cnt;
    int32_t *tris;                                       /* *3 */
} OrWorld;

enum { OR_VOL_POINT = 1, OR_VOL_SPHERE = 2, OR_VOL_BOX = 4, OR_VOL_REPLACE = 8, OR_VOL_STOP = 16 };

/* One full PhysicsWorld.step(dt) (world.py:410-430). Returns 0 or <0. */
int or_step(OrWorld *w);
/* Individual stages, for stage-level parity tests. */
void or_refit(OrWorld *w);                   /* world.py:471-508 */
int or_broadphase(OrWorld *w);               /* broadphase.py:243-294 */
void or_integrate_forces(OrWorld *w);        /* backend.py:26-40 */
void or_integrate_positions(OrWorld *w);     /* backend.py:42-49 */
/* Replace the warm-start cache with the given entries (copied). */
int or_set_cache(OrWorld *w, int32_t n, const int32_t *a, const int32_t *b,
                 const double *pt, const double *imp);
/* Free every oracle-owned buffer (outputs and cache). */
void or_free(OrWorld *w);

/* Narrowphase primitives on plain arrays (_collide_native.pyx:20-344,
 * gjk.py:249-264). R is row-major 3x3, columns = box axes. Return count. */
int or_box_box(const double *ca, const double *Ra, const double *ha,
               const double *cb, const double *Rb, const double *hb,
               double *normal, double *pts, double *depths);
int or_sphere_sphere(const double *ca, double ra, const double *cb, double rb,
                     double *normal, double *pts, double *depths);
int or_sphere_box(const double *cs, double rs, const double *cb, const double *Rb,
                  const double *hb, double *normal, double *pts, double *depths);
void or_quat_to_matrix(const double *q, double *R);   /* mathutil.py:59-76 */

/* capsule_triangles (_collide_native.pyx:454-574): the capsule segment
 * p0-p1 with radius against n triangles verts (n,3,3). hit[i] is written for
 * every triangle; points/normals/depths only where hit[i] = 1. */
void or_capsule_triangles(const double *p0, const double *p1, double radius,
                          const double *verts, int64_t n, uint8_t *hit,
                          double *points, double *normals, double *depths);

#ifdef __cplusplus
}
#endif
#endif
