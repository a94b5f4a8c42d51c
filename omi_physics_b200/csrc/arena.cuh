// Device arena: every world of a context, concatenated body-row ranges in a
// structure-of-arrays layout (the reference's numpy columns, world.py:75-122),
// plus the per-step scratch of each stage. Passed to kernels by value.
#pragma once
#include <cstdint>

namespace omi {

// per-contact prepared solver row (AoS, CD doubles, 16-byte multiple).
// The first C_PART doubles vary per contact (arms, effective masses, bias,
// depth); the rest is the same for every contact of one body pair (normal and
// tangent basis, friction, inverse masses, world inverse inertia of both
// bodies, the pair, dynamic flags), so a sweep loads it once per pair.
constexpr int CD = 44;
constexpr int C_PART = 12;
enum { C_RA = 0, C_RB = 3, C_NM = 6, C_T1M = 7, C_T2M = 8, C_VB = 9, C_DEPTH = 10,
       R_N = 12, R_T1 = 15, R_T2 = 18, R_FRIC = 21, R_IMA = 22, R_IMB = 23, R_IA = 24, R_IB = 33,
       R_AB = 42, R_FLAGS = 43 };
// per-joint prepared row: invIa(9) invIb(9) rA(3) rB(3) K/LU(9) piv(3) bias(3)
// n(3) mass bias_s
constexpr int JD = 48;
// narrowphase slot per pair: normal(3) + 4 x (point(3), depth)
constexpr int SLOT = 3 + 16;

// status words (device int array)
enum {
    ST_STEPS_DONE = 0,   // completed steps since the host last reset it
    ST_OVERFLOW = 1,     // 1 when a step found more pairs than pair_cap
    ST_PAIRS_NEEDED = 2, // pair count that overflowed
    ST_EPA_LIMIT = 3,    // EPA polytope exceeded its bounded storage
    ST_CASCADE = 4,      // wake cascades resolved sequentially (diagnostic)
    ST_GJK_ITEMS = 5,    // convex pairs routed to GJK/EPA in the last step
    ST_CONTACTS_NEEDED = 6,
    ST_SWEEP_TIMEOUT = 7, // a sweep wait ran out (never expected; the step is reported failed)
    ST_BOUNDS = 8,       // bounds-checked build: failed index checks (the accesses were skipped)
    ST_BOUNDS_SITE = 9,  // the first failed check: its site (BoundsSite)
    ST_BOUNDS_INDEX = 10, // ... and the index it refused
    ST_WORDS = 11
};

// Sites of the bounds-checked build's index checks (-DOMI_BOUNDS_CHECK,
// `_omi_b200_checked.so`): indices a kernel takes from data rather than from
// its own loop bounds, before the access they guard.
enum BoundsSite {
    BS_PAIR_BODY = 1,     // a candidate pair's body (narrowphase)
    BS_SHAPE = 2,         // a body's shape, and a hull's point range (GJK/EPA proxies)
    BS_CONTACT_BODY = 3,  // a contact's body (solver prep)
    BS_SWEEP_BODY = 4,    // a solver row's body, outside its world's staged rows (contact sweep)
    BS_SWEEP_RUN = 5,     // a successor run of a sweep entry (contact sweep)
    BS_JOINT_BODY = 6,    // a joint's body (joints)
    BS_ISLAND_BODY = 7,   // a contact body outside its world (islands and sleep)
    BS_FILTER_ROW = 8,    // a filter-matrix row (broadphase windows)
};

// In the bounds-checked build, OMI_BOUNDS(A, i, n, site, on_fail) checks
// 0 <= i < n; a failed check counts itself in ST_BOUNDS (the first one also
// records its site and index) and runs on_fail - a `continue`, `return` or
// assignment that skips the guarded access. It never traps: the host reports
// the step as failed (OMI_E_BOUNDS). In the shipped build the macro expands to
// nothing, so its device code is exactly the unchecked code.
#ifdef OMI_BOUNDS_CHECK
#define OMI_BOUNDS(A, i, n, site, on_fail) \
    if (!::omi::bounds_ok((A).status, (long long)(i), (long long)(n), (site))) { on_fail; }
#else
#define OMI_BOUNDS(A, i, n, site, on_fail)
#endif
#ifdef __CUDACC__
__device__ __forceinline__ bool bounds_ok(int *status, long long i, long long n, int site) {
    if (i >= 0 && i < n) return true;
    if (atomicAdd(&status[ST_BOUNDS], 1) == 0) {
        status[ST_BOUNDS_SITE] = site;
        status[ST_BOUNDS_INDEX] = (int)i;
    }
    return false;
}
#endif

// default bounds of the device's waits and of the EPA polytope; a context may
// lower them (omi_set_limits) so that a test can make them run out
constexpr int SPIN_LIMIT_DEFAULT = 1 << 22;


struct Arena {
    int W, NB, NS, NM, NJ, NPTS;
    int pair_cap, contact_cap, hash_mask;
    int spin_limit;                 // polls before a sweep wait gives up (ST_SWEEP_TIMEOUT)
    int epa_faces;                  // EPA polytope face bound (<= EPA_F; ST_EPA_LIMIT past it)
    int stall_run;                  // test hook: world-local run whose sweep entries never become ready (-1: none)
    int sweep_claim;                // ready sweep entries a warp claims at once (1-32; launch configuration)
    // wide worlds: large worlds whose stages run on many blocks (wide.cuh) instead of one
    // block per world; the per-world kernels skip them
    int n_wide;
    const int *wide_w;              // the wide worlds
    const uint8_t *w_wide;          // per world: 1 when wide
    int *wide_state;                // per wide world: WIDE_STATE_INTS ints of sweep counters
    int *wl_flag, *wl_scan;         // per contact: run-start flag and its scan (contact_cap + 1)
    int *wl_cnt, *wl_bstart;        // per body: run-bucket counts and their scan (NB + 1)
    int *wl_list;                   // run buckets of the wide worlds (2 * contact_cap)
    int *k_total;                   // contacts of the step (all worlds), the length of the run-start scan

    // worlds
    const int *w_body_off;          // row range of each world (its capacity)
    const int *w_body_n;            // live rows of each world (<= capacity)
    const int *w_joint_n;           // live joints of each world
    const double *w_g, *w_dt;
    const int *w_iters, *w_jiters;
    const int *w_flags;
    const uint8_t *w_active;
    const double *w_def_damp, *w_solver;
    const int *w_filter_off, *w_filter_rows, *w_pf_off, *w_pf_n, *w_joint_off;
    // gravity volumes (gravity.py:51-108): rows [w_vol_off[w], w_vol_off[w+1])
    // in application order; kind flags OMI_VOL_*, field = directional
    // acceleration or point centre, rc/rr = region centre, radius^2 / half
    const int *w_vol_off, *vol_kind;
    const double *vol_g, *vol_field, *vol_rc, *vol_rr;

    // bodies
    double *pos, *q, *v, *w, *prev_pos, *prev_q;
    const double *inv_mass, *inv_inertia, *gf, *ld, *ad, *qd;
    double *timer;
    uint8_t *awake;
    const int *mtype, *shape, *material, *material_key, *filter_row, *body_world;
    const int8_t *kind;      // 0 no shape, 1 sphere, 2 box, 3 convex, 4 capsule, 5 triangle mesh (of rshape)
    const double *half;      // refit half extents (world.py:443-469)
    const int *tshape;       // sensor shape (triggers.py) or -1
    const int *rshape;       // the shape a body's AABB comes from: collider, else sensor
    double *aabb_min, *aabb_max, *invIw;

    // shapes / materials / filters
    const int *shape_type;
    const double *shape_radius, *shape_size;
    const int *pt_off, *pt_cnt;
    const double *points;
    const double *mat_dynf, *mat_rest;
    const int *mat_fcomb, *mat_rcomb;
    const int *pf_a, *pf_b;
    const double *pf_mu;
    const uint8_t *filter_matrix;

    // joints
    const int *j_type, *j_a, *j_b;
    const double *j_anchor, *j_anchor_b, *j_axis, *j_target, *j_max_force;
    double *j_local_a, *j_local_b, *j_length, *j_accum;
    uint8_t *j_has_local_a, *j_has_local_b, *j_has_length;
    double *j_data;
    int *j_level, *j_order, *j_level_start;

    // broadphase
    int *order;              // sorted global body index per row (per world range)
    double *sorted_x;
    double *srt_box;         // per sorted row: lo/hi x, y, z and 2 pad (8 doubles)
    int *srt_info;           // per sorted row: motion type (bits 0-1), solid collider (2), awake (3),
                             // sensor (4), filter row (5-)
    int *pair_end;           // per sorted row: end of its sweep window
    unsigned long long *pair_mask;  // per sorted row: kept bits of its first 64 window rows
    double *sort_k[2];
    int *sort_v[2];
    int *pair_cnt, *pair_scan;      // NB, NB+1
    int *pair_a, *pair_b;           // pair_cap
    uint8_t *pair_solid;            // 1 contact pair, 2 sensor pair (no contact), 3 contact pair with a
                                    // triangle mesh (contacts written by k_mesh_emit), 0 neither

    // narrowphase
    int *slot_cnt;                  // pair_cap (+1 scratch)
    double *slot;                   // pair_cap * SLOT
    int *gjk_list, *gjk_n;
    int *trig_list, *trig_n;        // sensor pairs this step (pair indices)
    int *mesh_list, *mesh_n;        // pairs with a triangle-mesh body this step
    // static and kinematic triangle-mesh bodies (body.py:155-212): per mesh its triangle rows
    // [mesh_tri_off[m], mesh_tri_off[m+1]), the reference's uniform grid
    // (trigrid.py: exact flag, grid shape (3); low (3), high (3), cell size)
    // and per triangle world vertices (9), bounds (6), cell range (6), big flag
    const int *body_mesh;           // per body: mesh row or -1
    const int *mesh_tri_off, *mesh_grid_i;
    const double *mesh_grid_d, *tri_verts, *tri_box;
    const int *tri_cells;
    const uint8_t *tri_big;
    const int *tri_idx;             // per triangle: vertex indices into the mesh shape's points
    const int *mesh_body_of;        // per mesh: its body
    int *trig_out;                  // per sensor pair: trigger, other, overlap (1/0, -1 no shape)
    int *clip_list, *clip_n;        // touching box-box pairs awaiting face clipping
    int *contact_scan;              // pair_cap + 1

    // contacts
    int *c_a, *c_b;
    double *c_pt, *c_n, *c_depth, *c_imp, *c_data;
    int *c_order;                   // per world: the sweep's work ring (when not in shared memory)
    int *w_levels;                  // critical path of each world's last sweep, in contact solves
    int *w_runs;                    // runs (consecutive contacts of one body pair) per world
    int *run_k, *run_n, *run_a, *run_b;   // per run: first contact (world-local), count, dynamic bodies (-1 otherwise)
    int *run_pa, *run_pb;           // per run and side: predecessor code (k_levels)
    int *run_sa, *run_sb;           // per run and side: successor code (k_levels)
    int *run_kn, *run_need;         // per run: first contact | count << 24; need counts (k_levels)
    int *run_done, *run_tend;       // per run: sweep arrivals, finish slot (when not in shared memory)
    int *lv_scratch;                // k_levels buckets of worlds too large for shared memory
    int *sweep_next;                // next schedule index the sweep blocks take (reset by k_levels)
    int max_passes;                 // sweep passes the level buffers are sized for (warm start + iterations)
    const int *w_sched;             // worlds ordered largest first (per-world kernels)

    // per-body scratch
    int *b_last, *b_parent, *b_island;
    int *b_flag;

    // warm-start cache (ping-pong) and its hash tables
    int *cache_a[2], *cache_b[2];
    double *cache_pt[2], *cache_imp[2];
    int *w_cache_off[2], *w_cache_n[2];
    unsigned long long *hkey[2];
    int *hval[2];                   // packed start, count (2 ints per slot)
    int *hused[2], *hused_n;        // slots written by each table's last build; [2] = to clear
    int *parity;                    // current cache buffer (device)
    int *w_cache_new;               // W+1 scan scratch

    // scan scratch
    int *scan_blocks;

    int *status;
};

__host__ __device__ inline bool world_active(const Arena &A, int w) {
    return A.w_active[w] != 0;
}

}  // namespace omi
