/*
 * Oracle (test infrastructure only) — sequential CPU restatement of
 * omi_physics PhysicsWorld.step, float64, one world.
 *
 * Arithmetic follows the reference operation by operation so that results
 * agree with it bit-for-bit wherever the reference's own order is fixed:
 *   - the Cython accelerators (_collide_native.pyx, _solver_native.pyx) are
 *     plain C double arithmetic, restated here in the same order;
 *   - numpy einsum('nij,nj->ni') and einsum('nij,nkj->nik') sum their three
 *     terms as (t0 + t2) + t1 (measured on numpy 2.3.5);
 *   - np.linalg.norm(x, axis=-1) sums squares left to right, no FMA;
 *   - BLAS-backed np.dot / matmul / vec@mat on 3-vectors accumulate as the
 *     FMA chain fma(a2,b2, fma(a1,b1, a0*b0)); matrix@vector (gemv, no
 *     transpose) as fma(a2,b2, fma(a0,b0, a1*b1)) (numpy 2.3.5 + its bundled
 *     OpenBLAS, measured). These matter only on the GJK/EPA and joint paths.
 *   - np.linalg.solve (LAPACK dgesv) is restated as LU with partial pivoting;
 *     it agrees to ~1e-15 relative, not bit-for-bit.
 * Build with -ffp-contract=off (oracle/Makefile) so the compiler adds no FMA.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EPS_COLLIDE 1e-9   /* _collide_native.pyx:13, collide.py:34 */
#define EPS_GJK 1e-10      /* gjk.py:19 */

/* ------------------------------------------------------------------ */
/* small vector helpers                                                */
/* ------------------------------------------------------------------ */
static inline double dot_blas(const double *a, const double *b) {
    /* np.dot of two float64 3-vectors (BLAS ddot), see header comment */
    return fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0]));
}
static inline double gemv_row(const double *row, const double *x) {
    /* one row of M @ x for a C-contiguous 3x3 M (BLAS dgemv 'N') */
    return fma(row[2], x[2], fma(row[0], x[0], row[1] * x[1]));
}
static inline void cross_np(const double *a, const double *b, double *c) {
    /* np.cross (mathutil.py:79-87 / numpy): plain products */
    double x = a[1] * b[2] - a[2] * b[1];
    double y = a[2] * b[0] - a[0] * b[2];
    double z = a[0] * b[1] - a[1] * b[0];
    c[0] = x; c[1] = y; c[2] = z;
}
static inline double norm_axis3(const double *v) {
    /* np.linalg.norm(v, axis=-1): sqrt((x*x + y*y) + z*z) */
    return sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
}
static inline double norm_blas3(const double *v) {
    /* np.linalg.norm(v) with axis=None: sqrt(v.dot(v)) */
    return sqrt(dot_blas(v, v));
}
static inline void normalize3(const double *v, double *out) {
    /* mathutil.normalize (mathutil.py:21): v / max(norm, 1e-12) */
    double n = norm_axis3(v);
    double d = n > 1e-12 ? n : 1e-12;
    if (n != n) d = n;
    out[0] = v[0] / d; out[1] = v[1] / d; out[2] = v[2] / d;
}

/* mathutil.quat_to_matrix (mathutil.py:59-76), q is xyzw */
void or_quat_to_matrix(const double *qin, double *m) {
    double n = sqrt(((qin[0] * qin[0] + qin[1] * qin[1]) + qin[2] * qin[2]) + qin[3] * qin[3]);
    double d = n > 1e-12 ? n : 1e-12;
    if (n != n) d = n;
    double x = qin[0] / d, y = qin[1] / d, z = qin[2] / d, w = qin[3] / d;
    double xx = x * x, yy = y * y, zz = z * z;
    double xy = x * y, xz = x * z, yz = y * z;
    double wx = w * x, wy = w * y, wz = w * z;
    m[0] = 1.0 - 2.0 * (yy + zz);
    m[1] = 2.0 * (xy - wz);
    m[2] = 2.0 * (xz + wy);
    m[3] = 2.0 * (xy + wz);
    m[4] = 1.0 - 2.0 * (xx + zz);
    m[5] = 2.0 * (yz - wx);
    m[6] = 2.0 * (xz - wy);
    m[7] = 2.0 * (yz + wx);
    m[8] = 1.0 - 2.0 * (xx + yy);
}

/* world.py:_inv_inertia_world_all / solver.py:215-220:
 * invIw[i][k] = sum_j R[i][j]*invI[j]*R[k][j], einsum order (t0+t2)+t1 */
static void inv_inertia_world_einsum(const double *R, const double *invI, double *W) {
    double s[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) s[i * 3 + j] = R[i * 3 + j] * invI[j];
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++)
            W[i * 3 + k] = (s[i * 3 + 0] * R[k * 3 + 0] + s[i * 3 + 2] * R[k * 3 + 2]) +
                           s[i * 3 + 1] * R[k * 3 + 1];
}

/* joints.py:278-283: (R * invI) @ R.T through BLAS dgemm */
static void inv_inertia_world_gemm(const double *R, const double *invI, double *W) {
    double s[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) s[i * 3 + j] = R[i * 3 + j] * invI[j];
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) W[i * 3 + k] = dot_blas(&s[i * 3], &R[k * 3]);
}

static double combine_val(double a, double b, int mode) {
    /* model.combine (model.py:231-243) */
    if (mode == OR_MINIMUM) return b < a ? b : a;   /* Python min(a, b) */
    if (mode == OR_MAXIMUM) return b > a ? b : a;   /* Python max(a, b) */
    if (mode == OR_MULTIPLY) return a * b;
    return 0.5 * (a + b);
}

/* ------------------------------------------------------------------ */
/* growable buffers                                                    */
/* ------------------------------------------------------------------ */
static void *grow(void *p, size_t elem, int32_t need, int32_t *cap) {
    if (need <= *cap) return p;
    int32_t nc = *cap ? *cap : 64;
    while (nc < need) nc *= 2;
    void *q = realloc(p, (size_t)nc * elem);
    if (!q) return NULL;
    *cap = nc;
    return q;
}

typedef struct {
    int32_t pair_cap, solid_cap, contact_cap, cache_cap, overlap_cap;
} Caps;
static Caps g_caps_dummy;

/* Per-world capacity bookkeeping lives beside the OrWorld pointer. */
typedef struct CapEntry { const OrWorld *w; Caps c; struct CapEntry *next; } CapEntry;
static CapEntry *g_caps = NULL;
static Caps *caps_for(const OrWorld *w) {
    for (CapEntry *e = g_caps; e; e = e->next)
        if (e->w == w) return &e->c;
    CapEntry *e = (CapEntry *)calloc(1, sizeof(CapEntry));
    if (!e) return &g_caps_dummy;
    e->w = w; e->next = g_caps; g_caps = e;
    return &e->c;
}

/* ------------------------------------------------------------------ */
/* refit (world.py:443-508)                                            */
/* ------------------------------------------------------------------ */
static inline int trigger_of(const OrWorld *w, int i) {
    return w->trigger_shape ? w->trigger_shape[i] : -1;
}

/* the shape a body's AABB comes from: its collider, else its trigger
 * (world.py:452-455, 502-505) */
static int refit_shape(const OrWorld *w, int i) {
    int si = w->collider_shape[i];
    if (si >= 0 && si < w->n_shapes) return si;
    int ti = trigger_of(w, i);
    return (ti >= 0 && ti < w->n_shapes) ? ti : -1;
}

static int refit_kind(const OrWorld *w, int i) {
    int si = refit_shape(w, i);
    if (si < 0) return 0;
    int t = w->shape_type[si];
    if (t == OR_SHAPE_SPHERE) return 1;
    if (t == OR_SHAPE_BOX) return 2;
    return 3;
}

static void refit_half(const OrWorld *w, int i, double *half) {
    int si = refit_shape(w, i);
    half[0] = half[1] = half[2] = 0.0;
    if (si < 0) return;
    if (w->shape_type[si] == OR_SHAPE_SPHERE) {
        half[0] = half[1] = half[2] = w->shape_radius[si];
    } else if (w->shape_type[si] == OR_SHAPE_BOX) {
        for (int c = 0; c < 3; c++) half[c] = 0.5 * w->shape_size[si * 3 + c];
    }
}

/* CapsuleProxy segment ends (body.py:84-91): axis = R @ (0, 1, 0),
 * p0 = center - axis * half_height, p1 = center + axis * half_height */
static void capsule_ends(const double *center, const double *R, double hh, double *p0, double *p1) {
    static const double y[3] = {0.0, 1.0, 0.0};
    for (int c = 0; c < 3; c++) {
        double a = gemv_row(&R[c * 3], y) * hh;
        p0[c] = center[c] - a;
        p1[c] = center[c] + a;
    }
}

/* ConvexProxy world points (body.py:111-119): local @ R.T + center */
static void convex_world_points(const OrWorld *w, int si, const double *center,
                                const double *R, double *out) {
    int off = w->shape_pt_off[si], cnt = w->shape_pt_cnt[si];
    for (int p = 0; p < cnt; p++) {
        const double *l = &w->points[(off + p) * 3];
        for (int c = 0; c < 3; c++)
            out[p * 3 + c] = dot_blas(l, &R[c * 3]) + center[c];
    }
}

void or_refit(OrWorld *w) {
    double margin = w->margin;
    for (int i = 0; i < w->n; i++) {
        double R[9], half[3], hw[3];
        const double *pos = &w->pos[i * 3];
        or_quat_to_matrix(&w->q[i * 4], R);
        refit_half(w, i, half);
        int kind = refit_kind(w, i);
        for (int r = 0; r < 3; r++)
            hw[r] = (fabs(R[r * 3 + 0]) * half[0] + fabs(R[r * 3 + 2]) * half[2]) +
                    fabs(R[r * 3 + 1]) * half[1];
        if (kind == 1) { hw[0] = half[0]; hw[1] = half[1]; hw[2] = half[2]; }
        for (int c = 0; c < 3; c++) {
            w->aabb_min[i * 3 + c] = (pos[c] - hw[c]) - margin;
            w->aabb_max[i * 3 + c] = (pos[c] + hw[c]) + margin;
        }
        if (kind == 0) {
            for (int c = 0; c < 3; c++) w->aabb_min[i * 3 + c] = w->aabb_max[i * 3 + c] = pos[c];
        } else if (kind == 3 && w->shape_type[refit_shape(w, i)] == OR_SHAPE_CAPSULE) {
            /* CapsuleProxy.aabb (body.py:84-98) through world_aabb: segment
             * ends min/max -+ radius, then the refit margin */
            int si = refit_shape(w, i);
            double p0[3], p1[3];
            capsule_ends(pos, R, 0.5 * w->shape_size[si * 3 + 1], p0, p1);
            const double r = w->shape_radius[si];
            for (int c = 0; c < 3; c++) {
                double lo = p0[c] < p1[c] ? p0[c] : p1[c];
                double hi = p0[c] > p1[c] ? p0[c] : p1[c];
                w->aabb_min[i * 3 + c] = (lo - r) - margin;
                w->aabb_max[i * 3 + c] = (hi + r) + margin;
            }
        } else if (kind == 3) {
            int si = refit_shape(w, i);
            int cnt = w->shape_pt_cnt[si];
            double *pts = (double *)malloc(sizeof(double) * 3 * (cnt > 0 ? cnt : 1));
            convex_world_points(w, si, pos, R, pts);
            for (int c = 0; c < 3; c++) {
                double lo = pts[c], hi = pts[c];
                for (int p = 1; p < cnt; p++) {
                    double x = pts[p * 3 + c];
                    if (x < lo) lo = x;
                    if (x > hi) hi = x;
                }
                w->aabb_min[i * 3 + c] = lo - margin;
                w->aabb_max[i * 3 + c] = hi + margin;
            }
            free(pts);
        }
    }
}

/* ------------------------------------------------------------------ */
/* broadphase (broadphase.py:243-301)                                  */
/* ------------------------------------------------------------------ */
/* np.argsort(kind='stable') order: NaN after every number (+inf included),
 * -0.0 equal to 0.0, ties (NaNs among themselves too) by original index */
static const double *g_sort_keys;
static int cmp_stable(const void *pa, const void *pb) {
    int a = *(const int *)pa, b = *(const int *)pb;
    double ka = g_sort_keys[a * 3], kb = g_sort_keys[b * 3];
    int na = ka != ka, nb = kb != kb;
    if (na != nb) return na - nb;
    if (!na) {
        if (ka < kb) return -1;
        if (ka > kb) return 1;
    }
    return (a > b) - (a < b);   /* stable: original index breaks ties */
}

static int filters_interact(const OrWorld *w, int a, int b) {
    int nf = w->n_filters;
    int fa = w->collider_filter[a], fb = w->collider_filter[b];
    int ra = (fa >= 0 && fa < nf) ? fa + 1 : 0;
    int rb = (fb >= 0 && fb < nf) ? fb + 1 : 0;
    return w->filter_matrix ? w->filter_matrix[ra * (nf + 1) + rb] : 1;
}

int or_broadphase(OrWorld *w) {
    Caps *cp = caps_for(w);
    int n = w->n;
    w->n_pairs = 0;
    if (n < 2) return 0;
    int *order = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; i++) order[i] = i;
    g_sort_keys = w->aabb_min;
    qsort(order, n, sizeof(int), cmp_stable);
    for (int k = 0; k < n; k++) {
        int a = order[k];
        double hx = w->aabb_max[a * 3];
        /* searchsorted(lo_sx, hi_sx[k], 'right'): first index with lo > hi in
         * numpy's order, where NaN is above every number and equal to NaN: a NaN
         * row is past every finite hi, and a NaN hi is past every row */
        int lo = 0, hi = n;
        if (hx != hx) lo = n;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (w->aabb_min[order[mid] * 3] <= hx) lo = mid + 1; else hi = mid;
        }
        int end = lo;
        for (int kj = k + 1; kj < end; kj++) {
            int b = order[kj];
            const double *la = &w->aabb_min[a * 3], *ha = &w->aabb_max[a * 3];
            const double *lb = &w->aabb_min[b * 3], *hb = &w->aabb_max[b * 3];
            int keep = (ha[1] >= lb[1]) & (hb[1] >= la[1]) & (ha[2] >= lb[2]) & (hb[2] >= la[2]);
            keep &= (w->motion_type[a] == 2) | (w->motion_type[b] == 2);
            if (!keep) continue;
            int p = a < b ? a : b, qq = a < b ? b : a;
            if (!filters_interact(w, p, qq)) continue;
            w->pairs = (int32_t *)grow(w->pairs, sizeof(int32_t) * 2, w->n_pairs + 1, &cp->pair_cap);
            if (!w->pairs) { free(order); return -1; }
            w->pairs[w->n_pairs * 2] = p;
            w->pairs[w->n_pairs * 2 + 1] = qq;
            w->n_pairs++;
        }
    }
    free(order);
    return 0;
}

/* ------------------------------------------------------------------ */
/* box-box (_collide_native.pyx:20-263)                                */
/* ------------------------------------------------------------------ */
static int face_axis(const double *R, const double *dir, double *sign) {
    double best = -1.0;
    int axis = 0;
    for (int m = 0; m < 3; m++) {
        double dv = R[0 * 3 + m] * dir[0] + R[1 * 3 + m] * dir[1] + R[2 * 3 + m] * dir[2];
        if (fabs(dv) > best) {
            best = fabs(dv);
            axis = m;
            *sign = dv >= 0.0 ? 1.0 : -1.0;
        }
    }
    return axis;
}

static void face_vertices(const double *c, const double *R, const double *half, int axis,
                          double sign, double *verts) {
    int o0, o1;
    if (axis == 0) { o0 = 1; o1 = 2; }
    else if (axis == 1) { o0 = 0; o1 = 2; }
    else { o0 = 0; o1 = 1; }
    double fc[3], u[3], v[3];
    for (int r = 0; r < 3; r++) {
        fc[r] = c[r] + R[r * 3 + axis] * sign * half[axis];
        u[r] = R[r * 3 + o0] * half[o0];
        v[r] = R[r * 3 + o1] * half[o1];
    }
    for (int r = 0; r < 3; r++) {
        verts[0 * 3 + r] = fc[r] + u[r] + v[r];
        verts[1 * 3 + r] = fc[r] - u[r] + v[r];
        verts[2 * 3 + r] = fc[r] - u[r] - v[r];
        verts[3 * 3 + r] = fc[r] + u[r] - v[r];
    }
}

static int reduce_manifold(const double *allpts, const double *alldep, int nc,
                           double *out_pts, double *out_dep) {
    if (nc <= 4) {
        for (int i = 0; i < nc; i++) {
            for (int r = 0; r < 3; r++) out_pts[i * 3 + r] = allpts[i * 3 + r];
            out_dep[i] = alldep[i];
        }
        return nc;
    }
    int keep[4];
    double best = allpts[0];
    keep[0] = 0;
    for (int i = 1; i < nc; i++)
        if (allpts[i * 3] > best) { best = allpts[i * 3]; keep[0] = i; }
    keep[1] = 0; best = -1.0;
    for (int i = 0; i < nc; i++) {
        double dd = 0.0;
        for (int r = 0; r < 3; r++) {
            double d0 = allpts[i * 3 + r] - allpts[keep[0] * 3 + r];
            dd += d0 * d0;
        }
        if (dd > best) { best = dd; keep[1] = i; }
    }
    keep[2] = 0; best = -1.0;
    for (int i = 0; i < nc; i++) {
        double dsum = 0.0, dd = 0.0;
        for (int r = 0; r < 3; r++) {
            double d0 = allpts[i * 3 + r] - allpts[keep[1] * 3 + r];
            dsum += d0 * d0;
            d0 = allpts[i * 3 + r] - allpts[keep[0] * 3 + r];
            dd += d0 * d0;
        }
        if (sqrt(dsum) + sqrt(dd) > best) { best = sqrt(dsum) + sqrt(dd); keep[2] = i; }
    }
    keep[3] = 0; best = -1.0;
    for (int i = 0; i < nc; i++) {
        double dd = 0.0;
        for (int r = 0; r < 3; r++) {
            double d0 = allpts[i * 3 + r] - allpts[keep[2] * 3 + r];
            dd += d0 * d0;
        }
        if (sqrt(dd) > best) { best = sqrt(dd); keep[3] = i; }
    }
    int nk = 0;
    for (int i = 0; i < 4; i++) {
        int dup = 0;
        for (int j = 0; j < nk; j++)
            if (keep[i] == keep[j]) { dup = 1; break; }
        if (!dup) keep[nk++] = keep[i];
    }
    for (int i = 0; i < nk; i++) {
        for (int r = 0; r < 3; r++) out_pts[i * 3 + r] = allpts[keep[i] * 3 + r];
        out_dep[i] = alldep[keep[i]];
    }
    return nk;
}

static int clip_manifold(const double *ca, const double *Ra, const double *ha,
                         const double *cb, const double *Rb, const double *hb,
                         const double *normal, double depth, double *out_pts, double *out_dep) {
    double a_align = -1.0, b_align = -1.0;
    for (int m = 0; m < 3; m++) {
        double dv = fabs(Ra[0 * 3 + m] * normal[0] + Ra[1 * 3 + m] * normal[1] + Ra[2 * 3 + m] * normal[2]);
        if (dv > a_align) a_align = dv;
        dv = fabs(Rb[0 * 3 + m] * normal[0] + Rb[1 * 3 + m] * normal[1] + Rb[2 * 3 + m] * normal[2]);
        if (dv > b_align) b_align = dv;
    }
    const double *rc, *rR, *rh, *ic, *iR, *ih;
    int flip;
    if (a_align >= b_align) { rc = ca; rR = Ra; rh = ha; ic = cb; iR = Rb; ih = hb; flip = 0; }
    else { rc = cb; rR = Rb; rh = hb; ic = ca; iR = Ra; ih = ha; flip = 1; }
    double ref_n[3], neg[3];
    for (int r = 0; r < 3; r++) ref_n[r] = flip ? -normal[r] : normal[r];
    for (int r = 0; r < 3; r++) neg[r] = -ref_n[r];
    double isign = 0.0, rsign = 0.0;
    int iaxis = face_axis(iR, neg, &isign);
    double poly[16 * 3], buf[16 * 3];
    int np_ = 4;
    face_vertices(ic, iR, ih, iaxis, isign, poly);
    int raxis = face_axis(rR, ref_n, &rsign);
    double refv[12];
    face_vertices(rc, rR, rh, raxis, rsign, refv);
    double fp[3] = {refv[0], refv[1], refv[2]};
    for (int other = 0; other < 3 && np_ > 0; other++) {
        if (other == raxis) continue;
        for (int si = 0; si < 2; si++) {
            double s = si == 0 ? 1.0 : -1.0;
            double pn[3] = {rR[0 * 3 + other] * s, rR[1 * 3 + other] * s, rR[2 * 3 + other] * s};
            double offset = (rc[0] * pn[0] + rc[1] * pn[1] + rc[2] * pn[2]) + rh[other];
            int nb = 0;
            for (int i = 0; i < np_; i++) {
                const double *cur = &poly[i * 3], *nxt = &poly[((i + 1) % np_) * 3];
                double dc = pn[0] * cur[0] + pn[1] * cur[1] + pn[2] * cur[2] - offset;
                double dn = pn[0] * nxt[0] + pn[1] * nxt[1] + pn[2] * nxt[2] - offset;
                if (dc <= 0.0) {
                    buf[nb * 3] = cur[0]; buf[nb * 3 + 1] = cur[1]; buf[nb * 3 + 2] = cur[2];
                    nb++;
                }
                if (dc * dn < 0.0) {
                    double t = dc / (dc - dn);
                    for (int r = 0; r < 3; r++) buf[nb * 3 + r] = cur[r] + t * (nxt[r] - cur[r]);
                    nb++;
                }
            }
            np_ = nb;
            memcpy(poly, buf, sizeof(double) * 3 * nb);
            if (np_ == 0) break;
        }
    }
    double allpts[16 * 3], alldep[16];
    int nc = 0;
    for (int i = 0; i < np_; i++) {
        const double *p = &poly[i * 3];
        double pen = (fp[0] - p[0]) * ref_n[0] + (fp[1] - p[1]) * ref_n[1] + (fp[2] - p[2]) * ref_n[2];
        if (pen >= -1e-6) {
            for (int r = 0; r < 3; r++) allpts[nc * 3 + r] = p[r] + ref_n[r] * pen;
            alldep[nc] = pen > 0.0 ? pen : 0.0;
            nc++;
        }
    }
    if (nc == 0) {
        for (int r = 0; r < 3; r++) out_pts[r] = 0.5 * (ca[r] + cb[r]);
        out_dep[0] = depth;
        return 1;
    }
    return reduce_manifold(allpts, alldep, nc, out_pts, out_dep);
}

int or_box_box(const double *ca, const double *Ra, const double *ha,
               const double *cb, const double *Rb, const double *hb,
               double *normal, double *pts, double *depths) {
    double axes[15][3];
    int nax = 0;
    for (int i = 0; i < 3; i++) {
        axes[nax][0] = Ra[i]; axes[nax][1] = Ra[3 + i]; axes[nax][2] = Ra[6 + i]; nax++;
    }
    for (int i = 0; i < 3; i++) {
        axes[nax][0] = Rb[i]; axes[nax][1] = Rb[3 + i]; axes[nax][2] = Rb[6 + i]; nax++;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double cx = Ra[3 + i] * Rb[6 + j] - Ra[6 + i] * Rb[3 + j];
            double cy = Ra[6 + i] * Rb[0 + j] - Ra[0 + i] * Rb[6 + j];
            double cz = Ra[0 + i] * Rb[3 + j] - Ra[3 + i] * Rb[0 + j];
            double ln2 = cx * cx + cy * cy + cz * cz;
            if (ln2 > EPS_COLLIDE * EPS_COLLIDE) {
                double inv = 1.0 / sqrt(ln2);
                axes[nax][0] = cx * inv; axes[nax][1] = cy * inv; axes[nax][2] = cz * inv; nax++;
            }
        }
    double d[3] = {cb[0] - ca[0], cb[1] - ca[1], cb[2] - ca[2]};
    double best_depth = 1e300, best_axis[3] = {0.0, 0.0, 0.0};
    normal[0] = normal[1] = normal[2] = 0.0;
    for (int k = 0; k < nax; k++) {
        const double *ax = axes[k];
        double ra = (fabs(ax[0] * Ra[0] + ax[1] * Ra[3] + ax[2] * Ra[6]) * ha[0] +
                     fabs(ax[0] * Ra[1] + ax[1] * Ra[4] + ax[2] * Ra[7]) * ha[1] +
                     fabs(ax[0] * Ra[2] + ax[1] * Ra[5] + ax[2] * Ra[8]) * ha[2]);
        double rb = (fabs(ax[0] * Rb[0] + ax[1] * Rb[3] + ax[2] * Rb[6]) * hb[0] +
                     fabs(ax[0] * Rb[1] + ax[1] * Rb[4] + ax[2] * Rb[7]) * hb[1] +
                     fabs(ax[0] * Rb[2] + ax[1] * Rb[5] + ax[2] * Rb[8]) * hb[2]);
        double proj = ax[0] * d[0] + ax[1] * d[1] + ax[2] * d[2];
        double overlap = ra + rb - fabs(proj);
        if (overlap < 0.0) return 0;
        if (overlap < best_depth) {
            best_depth = overlap;
            double s = proj >= 0.0 ? 1.0 : -1.0;
            if (s > 0) { best_axis[0] = ax[0]; best_axis[1] = ax[1]; best_axis[2] = ax[2]; }
            else { best_axis[0] = -ax[0]; best_axis[1] = -ax[1]; best_axis[2] = -ax[2]; }
        }
    }
    normal[0] = best_axis[0]; normal[1] = best_axis[1]; normal[2] = best_axis[2];
    return clip_manifold(ca, Ra, ha, cb, Rb, hb, best_axis, best_depth, pts, depths);
}

/* _collide_native.pyx:285-299 */
int or_sphere_sphere(const double *ca, double ra, const double *cb, double rb,
                     double *normal, double *pts, double *depths) {
    double dx = cb[0] - ca[0], dy = cb[1] - ca[1], dz = cb[2] - ca[2];
    double dist = sqrt(dx * dx + dy * dy + dz * dz);
    double r = ra + rb;
    normal[0] = normal[1] = normal[2] = 0.0;
    if (dist >= r) return 0;
    double nx, ny, nz;
    if (dist > EPS_COLLIDE) { nx = dx / dist; ny = dy / dist; nz = dz / dist; }
    else { nx = 0.0; ny = 1.0; nz = 0.0; }
    double depth = r - dist;
    double f = ra - 0.5 * depth;
    normal[0] = nx; normal[1] = ny; normal[2] = nz;
    pts[0] = ca[0] + nx * f; pts[1] = ca[1] + ny * f; pts[2] = ca[2] + nz * f;
    depths[0] = depth;
    return 1;
}

/* _collide_native.pyx:302-344, normal returned sphere -> box */
int or_sphere_box(const double *cs, double rs, const double *cb, const double *Rb,
                  const double *hb, double *normal, double *pts, double *depths) {
    double sx = cs[0] - cb[0], sy = cs[1] - cb[1], sz = cs[2] - cb[2];
    double lx = Rb[0] * sx + Rb[3] * sy + Rb[6] * sz;
    double ly = Rb[1] * sx + Rb[4] * sy + Rb[7] * sz;
    double lz = Rb[2] * sx + Rb[5] * sy + Rb[8] * sz;
    double cx = lx, cy = ly, cz = lz;
    if (cx > hb[0]) cx = hb[0]; else if (cx < -hb[0]) cx = -hb[0];
    if (cy > hb[1]) cy = hb[1]; else if (cy < -hb[1]) cy = -hb[1];
    if (cz > hb[2]) cz = hb[2]; else if (cz < -hb[2]) cz = -hb[2];
    double dx = lx - cx, dy = ly - cy, dz = lz - cz;
    double dist = sqrt(dx * dx + dy * dy + dz * dz);
    normal[0] = normal[1] = normal[2] = 0.0;
    if (dist > rs) return 0;
    double nlx, nly, nlz, depth;
    if (dist > EPS_COLLIDE) {
        nlx = dx / dist; nly = dy / dist; nlz = dz / dist;
        depth = rs - dist;
    } else {
        double m0 = hb[0] - (lx >= 0 ? lx : -lx);
        double m1 = hb[1] - (ly >= 0 ? ly : -ly);
        double m2 = hb[2] - (lz >= 0 ? lz : -lz);
        int axis = 0;
        double mm = m0;
        if (m1 < mm) { axis = 1; mm = m1; }
        if (m2 < mm) { axis = 2; mm = m2; }
        nlx = nly = nlz = 0.0;
        if (axis == 0) nlx = lx >= 0 ? 1.0 : -1.0;
        else if (axis == 1) nly = ly >= 0 ? 1.0 : -1.0;
        else nlz = lz >= 0 ? 1.0 : -1.0;
        depth = rs + mm;
    }
    double nx = Rb[0] * nlx + Rb[1] * nly + Rb[2] * nlz;
    double ny = Rb[3] * nlx + Rb[4] * nly + Rb[5] * nlz;
    double nz = Rb[6] * nlx + Rb[7] * nly + Rb[8] * nlz;
    pts[0] = cb[0] + Rb[0] * cx + Rb[1] * cy + Rb[2] * cz;
    pts[1] = cb[1] + Rb[3] * cx + Rb[4] * cy + Rb[5] * cz;
    pts[2] = cb[2] + Rb[6] * cx + Rb[7] * cy + Rb[8] * cz;
    normal[0] = -nx; normal[1] = -ny; normal[2] = -nz;
    depths[0] = depth;
    return 1;
}

/* ------------------------------------------------------------------ */
/* GJK / EPA on support proxies (gjk.py, body.py:33-132)               */
/* ------------------------------------------------------------------ */
typedef struct {
    int kind;             /* 1 sphere, 2 box, 3 convex, 4 capsule */
    double center[3], R[9], half[3], radius;
    double p0[3], p1[3];  /* capsule segment ends */
    const double *world;  /* convex world points */
    int m;
} Proxy;

static void proxy_support(const Proxy *p, const double *d, double *out) {
    if (p->kind == 1) {                         /* body.py:46-48 */
        double u[3];
        normalize3(d, u);
        for (int c = 0; c < 3; c++) out[c] = p->center[c] + p->radius * u[c];
    } else if (p->kind == 2) {                  /* body.py:69-73 */
        double local[3], s[3];
        for (int j = 0; j < 3; j++) {
            double col[3] = {p->R[j], p->R[3 + j], p->R[6 + j]};
            local[j] = dot_blas(col, d);
        }
        for (int j = 0; j < 3; j++) {
            double sg = local[j] > 0 ? 1.0 : (local[j] < 0 ? -1.0 : (local[j] == 0 ? 0.0 : local[j]));
            s[j] = sg * p->half[j];
        }
        for (int c = 0; c < 3; c++) out[c] = p->center[c] + gemv_row(&p->R[c * 3], s);
    } else if (p->kind == OR_SHAPE_CAPSULE) {   /* body.py:100-104 */
        const double *end = dot_blas(p->p0, d) > dot_blas(p->p1, d) ? p->p0 : p->p1;
        double u[3];
        normalize3(d, u);
        for (int c = 0; c < 3; c++) out[c] = end[c] + p->radius * u[c];
    } else {                                    /* body.py:125-128 */
        int best = 0;
        double bv = gemv_row(&p->world[0], d);
        for (int i = 1; i < p->m; i++) {
            double v = gemv_row(&p->world[i * 3], d);
            if (v > bv) { bv = v; best = i; }
        }
        for (int c = 0; c < 3; c++) out[c] = p->world[best * 3 + c];
    }
}

static void proxy_center_hint(const Proxy *p, double *out) {
    if (p->kind != 3) { for (int c = 0; c < 3; c++) out[c] = p->center[c]; return; }
    double s[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < p->m; i++)
        for (int c = 0; c < 3; c++) s[c] = s[c] + p->world[i * 3 + c];
    for (int c = 0; c < 3; c++) out[c] = s[c] / (double)p->m;
}

typedef struct { double v[3], a[3], b[3]; } Vtx;

static void mink_support(const Proxy *A, const Proxy *B, const double *d, Vtx *out) {
    double nd[3] = {-d[0], -d[1], -d[2]};
    proxy_support(A, d, out->a);
    proxy_support(B, nd, out->b);
    for (int c = 0; c < 3; c++) out->v[c] = out->a[c] - out->b[c];
}

static inline void sub3(const double *a, const double *b, double *c) {
    c[0] = a[0] - b[0]; c[1] = a[1] - b[1]; c[2] = a[2] - b[2];
}
static inline void neg3(const double *a, double *c) { c[0] = -a[0]; c[1] = -a[1]; c[2] = -a[2]; }

/* simplex stored as list order s[0..n-1] (gjk.py list order) */
static int gjk_line(Vtx *s, int *n, double *d) {
    Vtx b = s[0], a = s[1];
    double ab[3], ao[3];
    sub3(b.v, a.v, ab); neg3(a.v, ao);
    if (dot_blas(ab, ao) > 0) {
        double t[3];
        cross_np(ab, ao, t); cross_np(t, ab, d);
        if (dot_blas(d, d) < EPS_GJK) {           /* _any_perp, gjk.py:114-117 */
            double ax[3];
            if (fabs(ab[0]) < 0.9) { ax[0] = 1.0; ax[1] = 0.0; ax[2] = 0.0; }
            else { ax[0] = 0.0; ax[1] = 1.0; ax[2] = 0.0; }
            cross_np(ab, ax, d);
        }
        s[0] = b; s[1] = a; *n = 2;
        return 0;
    }
    s[0] = a; *n = 1;
    d[0] = ao[0]; d[1] = ao[1]; d[2] = ao[2];
    return 0;
}

static int gjk_triangle(Vtx *s, int *n, double *d) {
    Vtx c = s[0], b = s[1], a = s[2];
    double ab[3], ac[3], ao[3], abc[3], t[3];
    sub3(b.v, a.v, ab); sub3(c.v, a.v, ac); neg3(a.v, ao);
    cross_np(ab, ac, abc);
    cross_np(abc, ac, t);
    if (dot_blas(t, ao) > 0) {
        if (dot_blas(ac, ao) > 0) {
            double u[3];
            cross_np(ac, ao, u); cross_np(u, ac, d);
            s[0] = c; s[1] = a; *n = 2;
            return 0;
        }
        s[0] = b; s[1] = a; *n = 2;
        return gjk_line(s, n, d);
    }
    cross_np(ab, abc, t);
    if (dot_blas(t, ao) > 0) {
        s[0] = b; s[1] = a; *n = 2;
        return gjk_line(s, n, d);
    }
    if (dot_blas(abc, ao) > 0) {
        s[0] = c; s[1] = b; s[2] = a; *n = 3;
        d[0] = abc[0]; d[1] = abc[1]; d[2] = abc[2];
        return 0;
    }
    s[0] = b; s[1] = c; s[2] = a; *n = 3;
    neg3(abc, d);
    return 0;
}

static int gjk_tetra(Vtx *s, int *n, double *dir) {
    Vtx d = s[0], c = s[1], b = s[2], a = s[3];
    double ab[3], ac[3], ad[3], ao[3], abc[3], acd[3], adb[3];
    sub3(b.v, a.v, ab); sub3(c.v, a.v, ac); sub3(d.v, a.v, ad); neg3(a.v, ao);
    cross_np(ab, ac, abc); cross_np(ac, ad, acd); cross_np(ad, ab, adb);
    if (dot_blas(abc, ao) > 0) { s[0] = c; s[1] = b; s[2] = a; *n = 3; return gjk_triangle(s, n, dir); }
    if (dot_blas(acd, ao) > 0) { s[0] = d; s[1] = c; s[2] = a; *n = 3; return gjk_triangle(s, n, dir); }
    if (dot_blas(adb, ao) > 0) { s[0] = b; s[1] = d; s[2] = a; *n = 3; return gjk_triangle(s, n, dir); }
    dir[0] = dir[1] = dir[2] = 0.0;
    return 1;
}

/* gjk.py:39-57 */
static int gjk_intersect(const Proxy *A, const Proxy *B, Vtx *s, int *n) {
    double zero[3] = {0.0, 0.0, 0.0}, pa[3], pb[3], d[3], nd[3];
    proxy_support(B, zero, pb);
    proxy_support(A, zero, pa);
    sub3(pb, pa, d);
    if (dot_blas(d, d) < EPS_GJK) { d[0] = 1.0; d[1] = 0.0; d[2] = 0.0; }
    neg3(d, nd);
    mink_support(A, B, nd, &s[0]);
    *n = 1;
    neg3(s[0].v, d);
    for (int it = 0; it < 32; it++) {
        if (dot_blas(d, d) < EPS_GJK) return 1;
        Vtx wv;
        mink_support(A, B, d, &wv);
        if (dot_blas(wv.v, d) < 0) return 0;
        s[(*n)++] = wv;
        int contains;
        if (*n == 2) contains = gjk_line(s, n, d);
        else if (*n == 3) contains = gjk_triangle(s, n, d);
        else contains = gjk_tetra(s, n, d);
        if (contains) return 1;
    }
    return 0;
}

#define EPA_MAX_V (4 + 64 + 1)
#define EPA_MAX_F 512
typedef struct { int i, j, k; } Face;

/* gjk.py:176-194 */
static int closest_face(const Vtx *V, const Face *F, int nf, double *bn, double *bd) {
    int best = -1;
    double best_d = INFINITY;
    for (int f = 0; f < nf; f++) {
        const double *a = V[F[f].i].v, *b = V[F[f].j].v, *c = V[F[f].k].v;
        double e1[3], e2[3], nrm[3];
        sub3(b, a, e1); sub3(c, a, e2);
        cross_np(e1, e2, nrm);
        double ln = norm_blas3(nrm);
        if (ln < EPS_GJK) continue;
        for (int q = 0; q < 3; q++) nrm[q] = nrm[q] / ln;
        double dd = dot_blas(nrm, a);
        if (dd < 0) { neg3(nrm, nrm); dd = -dd; }
        if (dd < best_d) { best = f; best_d = dd; bn[0] = nrm[0]; bn[1] = nrm[1]; bn[2] = nrm[2]; }
    }
    *bd = best_d;
    return best;
}

/* gjk.py:197-217 */
static int rebuild(const Vtx *V, Face *F, int nf, int ni) {
    const double *w = V[ni].v;
    int ei[3 * EPA_MAX_F], ej[3 * EPA_MAX_F];
    unsigned char alive[3 * EPA_MAX_F];
    int ne = 0, nk = 0;
    Face kept[EPA_MAX_F];
    for (int f = 0; f < nf; f++) {
        const double *a = V[F[f].i].v;
        double e1[3], e2[3], nrm[3], wa[3];
        sub3(V[F[f].j].v, a, e1); sub3(V[F[f].k].v, a, e2);
        cross_np(e1, e2, nrm);
        sub3(w, a, wa);
        if (dot_blas(nrm, wa) > 0) {
            int es[3][2] = {{F[f].i, F[f].j}, {F[f].j, F[f].k}, {F[f].k, F[f].i}};
            for (int e = 0; e < 3; e++) {
                int found_rev = -1, found = -1;
                for (int q = 0; q < ne; q++) {
                    if (!alive[q]) continue;
                    if (ei[q] == es[e][1] && ej[q] == es[e][0]) found_rev = q;
                    if (ei[q] == es[e][0] && ej[q] == es[e][1]) found = q;
                }
                if (found_rev >= 0) alive[found_rev] = 0;
                else if (found < 0) {
                    if (ne >= 3 * EPA_MAX_F) return -1;
                    ei[ne] = es[e][0]; ej[ne] = es[e][1]; alive[ne] = 1; ne++;
                }
            }
        } else {
            kept[nk++] = F[f];
        }
    }
    for (int q = 0; q < ne; q++) {
        if (!alive[q]) continue;
        if (nk >= EPA_MAX_F) return -1;
        kept[nk].i = ei[q]; kept[nk].j = ej[q]; kept[nk].k = ni; nk++;
    }
    memcpy(F, kept, sizeof(Face) * nk);
    return nk;
}

/* gjk.py:220-246 */
static void contact_from_face(const Vtx *V, Face f, const double *nrm, double dist, double *point) {
    const Vtx *a = &V[f.i], *b = &V[f.j], *c = &V[f.k];
    double p[3] = {nrm[0] * dist, nrm[1] * dist, nrm[2] * dist};
    double v0[3], v1[3], v2[3];
    sub3(b->v, a->v, v0); sub3(c->v, a->v, v1); sub3(p, a->v, v2);
    double d00 = dot_blas(v0, v0), d01 = dot_blas(v0, v1), d11 = dot_blas(v1, v1);
    double d20 = dot_blas(v2, v0), d21 = dot_blas(v2, v1);
    double denom = d00 * d11 - d01 * d01;
    double bu, bv, bw;
    if (fabs(denom) < EPS_GJK) { bu = 1.0; bv = 0.0; bw = 0.0; }
    else {
        bv = (d11 * d20 - d01 * d21) / denom;
        bw = (d00 * d21 - d01 * d20) / denom;
        bu = 1.0 - bv - bw;
    }
    for (int q = 0; q < 3; q++) {
        double pa = bu * a->a[q] + bv * b->a[q] + bw * c->a[q];
        double pb = bu * a->b[q] + bv * b->b[q] + bw * c->b[q];
        point[q] = 0.5 * (pa + pb);
    }
}

/* gjk.py:155-173 */
static int expand_to_tetra(const Proxy *A, const Proxy *B, Vtx *V, int *n) {
    static const double dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (int k = 0; k < 6; k++) {
        if (*n >= 4) break;
        Vtx wv;
        mink_support(A, B, dirs[k], &wv);
        int ok = 1;
        for (int p = 0; p < *n; p++) {
            double dv[3];
            sub3(wv.v, V[p].v, dv);
            if (!(dot_blas(dv, dv) > EPS_GJK)) { ok = 0; break; }
        }
        if (ok) V[(*n)++] = wv;
    }
    if (*n < 4) return 0;
    double e1[3], e2[3], e3[3], cr[3];
    sub3(V[1].v, V[0].v, e1); sub3(V[2].v, V[0].v, e2); sub3(V[3].v, V[0].v, e3);
    cross_np(e1, e2, cr);
    if (dot_blas(cr, e3) > 0) { Vtx t = V[1]; V[1] = V[2]; V[2] = t; }
    *n = 4;
    return 1;
}

/* gjk.py:120-152 */
static int epa(const Proxy *A, const Proxy *B, Vtx *V, int nv, double *nrm, double *depth,
               double *point) {
    static Face F[EPA_MAX_F];
    if (nv < 4) {
        if (!expand_to_tetra(A, B, V, &nv)) return 0;
    }
    int nf = 4;
    F[0] = (Face){0, 1, 2}; F[1] = (Face){0, 2, 3}; F[2] = (Face){0, 3, 1}; F[3] = (Face){1, 3, 2};
    for (int it = 0; it < 64; it++) {
        double bn[3], bd;
        int bf = closest_face(V, F, nf, bn, &bd);
        if (bf < 0) return 0;
        Vtx wv;
        mink_support(A, B, bn, &wv);
        double dd = dot_blas(wv.v, bn);
        if (dd - bd < 1e-6) {
            contact_from_face(V, F[bf], bn, bd, point);
            nrm[0] = bn[0]; nrm[1] = bn[1]; nrm[2] = bn[2]; *depth = bd;
            return 1;
        }
        V[nv++] = wv;
        nf = rebuild(V, F, nf, nv - 1);
        if (nf <= 0) return 0;
    }
    double bn[3], bd;
    int bf = closest_face(V, F, nf, bn, &bd);
    if (bf < 0) return 0;
    contact_from_face(V, F[bf], bn, bd, point);
    nrm[0] = bn[0]; nrm[1] = bn[1]; nrm[2] = bn[2]; *depth = bd;
    return 1;
}

/* gjk.collide_convex (gjk.py:249-264) */
static int collide_convex(const Proxy *A, const Proxy *B, double *normal, double *point,
                          double *depth) {
    Vtx V[EPA_MAX_V];
    int nv = 0;
    if (!gjk_intersect(A, B, V, &nv)) return 0;
    double nrm[3], dep, pt[3];
    if (!epa(A, B, V, nv, nrm, &dep, pt)) return 0;
    double ha[3], hb[3], dc[3];
    proxy_center_hint(A, ha); proxy_center_hint(B, hb);
    sub3(hb, ha, dc);
    if (dot_blas(nrm, dc) < 0) neg3(nrm, nrm);
    if (dep <= 1e-9) return 0;
    normalize3(nrm, normal);
    point[0] = pt[0]; point[1] = pt[1]; point[2] = pt[2];
    *depth = dep;
    return 1;
}

/* Test hook: gjk.collide_convex on two proxies given as plain arrays.
 * kind 1 sphere (r), 2 box (half), 3 convex (m local points),
 * 4 capsule (r, half[1] = half height). */
int or_collide_convex(int ka, const double *ca, const double *qa, const double *ha, double ra,
                      const double *pa, int ma, int kb, const double *cb, const double *qb,
                      const double *hb, double rb, const double *pb, int mb, double *normal,
                      double *point, double *depth) {
    Proxy A, B;
    double *wa = (double *)malloc(sizeof(double) * 3 * (ma > 0 ? ma : 1));
    double *wb = (double *)malloc(sizeof(double) * 3 * (mb > 0 ? mb : 1));
    const int ks[2] = {ka, kb};
    const double *cs[2] = {ca, cb}, *qs[2] = {qa, qb}, *hs[2] = {ha, hb}, *ps[2] = {pa, pb};
    const double rs[2] = {ra, rb};
    const int ms[2] = {ma, mb};
    Proxy *P[2] = {&A, &B};
    double *W[2] = {wa, wb};
    for (int e = 0; e < 2; e++) {
        Proxy *p = P[e];
        p->kind = ks[e];
        or_quat_to_matrix(qs[e], p->R);
        for (int c = 0; c < 3; c++) { p->center[c] = cs[e][c]; p->half[c] = hs[e][c]; }
        p->radius = rs[e];
        if (ks[e] == OR_SHAPE_CAPSULE) capsule_ends(p->center, p->R, p->half[1], p->p0, p->p1);
        p->m = ms[e];
        for (int i = 0; i < ms[e]; i++)
            for (int c = 0; c < 3; c++)
                W[e][i * 3 + c] = dot_blas(&ps[e][i * 3], &p->R[c * 3]) + p->center[c];
        p->world = W[e];
    }
    int r = collide_convex(&A, &B, normal, point, depth);
    free(wa); free(wb);
    return r;
}

/* make_proxy (body.py:214-237) of shape si at body i's pose */
static void make_proxy_shape(const OrWorld *w, int si, int i, Proxy *p, double *scratch) {
    int t = w->shape_type[si];
    or_quat_to_matrix(&w->q[i * 4], p->R);
    for (int c = 0; c < 3; c++) p->center[c] = w->pos[i * 3 + c];
    p->kind = t;
    if (t == OR_SHAPE_SPHERE) {
        p->radius = w->shape_radius[si];
    } else if (t == OR_SHAPE_BOX) {
        for (int c = 0; c < 3; c++) p->half[c] = 0.5 * w->shape_size[si * 3 + c];
    } else if (t == OR_SHAPE_CAPSULE) {         /* make_proxy (body.py:224-228) */
        p->radius = w->shape_radius[si];
        capsule_ends(p->center, p->R, 0.5 * w->shape_size[si * 3 + 1], p->p0, p->p1);
    } else {
        p->m = w->shape_pt_cnt[si];
        convex_world_points(w, si, p->center, p->R, scratch);
        p->world = scratch;
    }
}

static void make_proxy(const OrWorld *w, int i, Proxy *p, double *scratch) {
    make_proxy_shape(w, w->collider_shape[i], i, p, scratch);
}

/* ------------------------------------------------------------------ */
/* narrowphase (narrowphase.py:51-100) + solid filter (world.py:658-671) */
/* ------------------------------------------------------------------ */
static int awake_mover(const OrWorld *w, int i) {   /* world.py:381-384 */
    int t = w->motion_type[i];
    return (t == 2 && w->awake[i]) || t == 1;
}

static int push_contact(OrWorld *w, Caps *cp, int a, int b, const double *pt, const double *nrm,
                        double depth) {
    int k = w->n_contacts;
    int32_t cap = cp->contact_cap;
    w->c_a = (int32_t *)grow(w->c_a, sizeof(int32_t), k + 1, &cap);
    cap = cp->contact_cap;
    w->c_b = (int32_t *)grow(w->c_b, sizeof(int32_t), k + 1, &cap);
    cap = cp->contact_cap;
    w->c_pt = (double *)grow(w->c_pt, sizeof(double) * 3, k + 1, &cap);
    cap = cp->contact_cap;
    w->c_n = (double *)grow(w->c_n, sizeof(double) * 3, k + 1, &cap);
    cap = cp->contact_cap;
    w->c_depth = (double *)grow(w->c_depth, sizeof(double), k + 1, &cap);
    cap = cp->contact_cap;
    w->c_imp = (double *)grow(w->c_imp, sizeof(double) * 3, k + 1, &cap);
    cp->contact_cap = cap;
    if (!w->c_a || !w->c_b || !w->c_pt || !w->c_n || !w->c_depth || !w->c_imp) return -1;
    w->c_a[k] = a; w->c_b[k] = b;
    for (int c = 0; c < 3; c++) { w->c_pt[k * 3 + c] = pt[c]; w->c_n[k * 3 + c] = nrm[c]; }
    w->c_depth[k] = depth;
    w->c_imp[k * 3] = w->c_imp[k * 3 + 1] = w->c_imp[k * 3 + 2] = 0.0;
    w->n_contacts = k + 1;
    return 0;
}

static int collide_mesh(OrWorld *w, Caps *cp, int a, int b);
static int g_mesh_pass;

static int narrowphase(OrWorld *w) {
    g_mesh_pass++;                       /* mesh tables are rebuilt once per pass */
    Caps *cp = caps_for(w);
    w->n_solid = 0;
    w->n_contacts = 0;
    int maxpts = 1;
    for (int s = 0; s < w->n_shapes; s++)
        if ((w->shape_type[s] == OR_SHAPE_CONVEX || w->shape_type[s] == OR_SHAPE_TRIMESH) &&
            w->shape_pt_cnt[s] > maxpts) maxpts = w->shape_pt_cnt[s];
    double *sa = (double *)malloc(sizeof(double) * 3 * maxpts);
    double *sb = (double *)malloc(sizeof(double) * 3 * maxpts);
    for (int p = 0; p < w->n_pairs; p++) {
        int i = w->pairs[p * 2], j = w->pairs[p * 2 + 1];
        if (trigger_of(w, i) >= 0 || trigger_of(w, j) >= 0) continue;   /* trigger pairs: no contact */
        if (!(w->collider_shape[i] >= 0 && w->collider_shape[j] >= 0)) continue;
        if (!(awake_mover(w, i) || awake_mover(w, j))) continue;
        w->solid = (int32_t *)grow(w->solid, sizeof(int32_t) * 2, w->n_solid + 1, &cp->solid_cap);
        w->solid[w->n_solid * 2] = i;
        w->solid[w->n_solid * 2 + 1] = j;
        w->n_solid++;
    }
    for (int p = 0; p < w->n_solid; p++) {
        int a = w->solid[p * 2], b = w->solid[p * 2 + 1];
        int ka = refit_kind(w, a), kb = refit_kind(w, b);
        double Ra[9], Rb[9], ha[3], hb[3], nrm[3], pts[12], dep[4];
        int cnt = 0;
        const double *pa = &w->pos[a * 3], *pb = &w->pos[b * 3];
        or_quat_to_matrix(&w->q[a * 4], Ra);
        or_quat_to_matrix(&w->q[b * 4], Rb);
        refit_half(w, a, ha);
        refit_half(w, b, hb);
        if (ka == 2 && kb == 2) {
            cnt = or_box_box(pa, Ra, ha, pb, Rb, hb, nrm, pts, dep);
        } else if (ka == 1 && kb == 1) {
            cnt = or_sphere_sphere(pa, ha[0], pb, hb[0], nrm, pts, dep);
        } else if (ka == 1 && kb == 2) {
            cnt = or_sphere_box(pa, ha[0], pb, Rb, hb, nrm, pts, dep);
        } else if (ka == 2 && kb == 1) {
            cnt = or_sphere_box(pb, hb[0], pa, Ra, ha, nrm, pts, dep);
            nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
        } else if (w->shape_type[w->collider_shape[a]] == OR_SHAPE_TRIMESH ||
                   w->shape_type[w->collider_shape[b]] == OR_SHAPE_TRIMESH) {
            if (collide_mesh(w, cp, a, b)) { free(sa); free(sb); return -1; }
            continue;
        } else {
            Proxy A, B;
            make_proxy(w, a, &A, sa);
            make_proxy(w, b, &B, sb);
            cnt = collide_convex(&A, &B, nrm, pts, dep);
        }
        for (int k = 0; k < cnt; k++)
            if (push_contact(w, cp, a, b, &pts[k * 3], nrm, dep[k])) { free(sa); free(sb); return -1; }
    }
    free(sa); free(sb);
    return 0;
}

/* ------------------------------------------------------------------ */
/* contact solver (solver.py:192-337, _solver_native.pyx:132-312)     */
/* ------------------------------------------------------------------ */
static void wake(OrWorld *w, int i) { w->awake[i] = 1; w->sleep_timer[i] = 0.0; }

static void wake_sleepers(OrWorld *w) {
    double thr = 0.15 * 0.15;
    double *v2 = (double *)malloc(sizeof(double) * (w->n ? w->n : 1));
    for (int i = 0; i < w->n; i++) {
        const double *v = &w->v[i * 3];
        v2[i] = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
    }
    for (int k = 0; k < w->n_contacts; k++) {
        int a = w->c_a[k], b = w->c_b[k];
        int ta = w->motion_type[a], tb = w->motion_type[b];
        if (!w->awake[b]) {
            int wk = ta == 1 || (ta == 2 && w->awake[a] && v2[a] > thr);
            if (wk) wake(w, b);
        }
        if (!w->awake[a]) {
            int wk = tb == 1 || (tb == 2 && w->awake[b] && v2[b] > thr);
            if (wk) wake(w, a);
        }
    }
    free(v2);
}

static const OrWorld *g_mat_w;
static void material(const OrWorld *w, int i, double *dynf, double *rest, int *fc, int *rc) {
    int m = w->collider_material[i];
    if (m >= 0 && m < w->n_materials) {
        *dynf = w->mat_dynf[m]; *rest = w->mat_rest[m]; *fc = w->mat_fcomb[m]; *rc = w->mat_rcomb[m];
    } else {
        *dynf = 0.6; *rest = 0.0; *fc = OR_AVERAGE; *rc = OR_AVERAGE;   /* DEFAULT_MATERIAL */
    }
}

static int pair_friction(const OrWorld *w, int ma, int mb, double *mu) {
    int a = ma <= mb ? ma : mb, b = ma <= mb ? mb : ma;
    for (int p = 0; p < w->n_pair_friction; p++)
        if (w->pf_a[p] == a && w->pf_b[p] == b) { *mu = w->pf_mu[p]; return 1; }
    return 0;
}

static void apply_w(double *lv, double *av, int a, int b, double ima, double imb,
                    const double *invIw, const double *rA, const double *rB,
                    double Px, double Py, double Pz) {
    double crx, cry, crz;
    lv[a * 3 + 0] -= ima * Px; lv[a * 3 + 1] -= ima * Py; lv[a * 3 + 2] -= ima * Pz;
    lv[b * 3 + 0] += imb * Px; lv[b * 3 + 1] += imb * Py; lv[b * 3 + 2] += imb * Pz;
    const double *Ia = &invIw[a * 9], *Ib = &invIw[b * 9];
    crx = rA[1] * Pz - rA[2] * Py;
    cry = rA[2] * Px - rA[0] * Pz;
    crz = rA[0] * Py - rA[1] * Px;
    av[a * 3 + 0] -= Ia[0] * crx + Ia[1] * cry + Ia[2] * crz;
    av[a * 3 + 1] -= Ia[3] * crx + Ia[4] * cry + Ia[5] * crz;
    av[a * 3 + 2] -= Ia[6] * crx + Ia[7] * cry + Ia[8] * crz;
    crx = rB[1] * Pz - rB[2] * Py;
    cry = rB[2] * Px - rB[0] * Pz;
    crz = rB[0] * Py - rB[1] * Px;
    av[b * 3 + 0] += Ib[0] * crx + Ib[1] * cry + Ib[2] * crz;
    av[b * 3 + 1] += Ib[3] * crx + Ib[4] * cry + Ib[5] * crz;
    av[b * 3 + 2] += Ib[6] * crx + Ib[7] * cry + Ib[8] * crz;
}

static double effmass(const double *ra, const double *rb, double dx, double dy, double dz,
                      const double *invIw, int a, int b, double ima, double imb) {
    double ax = ra[1] * dz - ra[2] * dy, ay = ra[2] * dx - ra[0] * dz, az = ra[0] * dy - ra[1] * dx;
    double bx = rb[1] * dz - rb[2] * dy, by = rb[2] * dx - rb[0] * dz, bz = rb[0] * dy - rb[1] * dx;
    const double *Ia = &invIw[a * 9], *Ib = &invIw[b * 9];
    double kk = ima + imb;
    double wx = Ia[0] * ax + Ia[1] * ay + Ia[2] * az;
    double wy = Ia[3] * ax + Ia[4] * ay + Ia[5] * az;
    double wz = Ia[6] * ax + Ia[7] * ay + Ia[8] * az;
    kk += ax * wx + ay * wy + az * wz;
    wx = Ib[0] * bx + Ib[1] * by + Ib[2] * bz;
    wy = Ib[3] * bx + Ib[4] * by + Ib[5] * bz;
    wz = Ib[6] * bx + Ib[7] * by + Ib[8] * bz;
    kk += bx * wx + by * wy + bz * wz;
    return kk > 1e-12 ? 1.0 / kk : 0.0;
}

#define REL_VEL(lv, av, a, b, rA, rB, dvx, dvy, dvz)                                          \
    do {                                                                                      \
        dvx = (lv[b * 3 + 0] + av[b * 3 + 1] * rB[2] - av[b * 3 + 2] * rB[1]) -                \
              (lv[a * 3 + 0] + av[a * 3 + 1] * rA[2] - av[a * 3 + 2] * rA[1]);                 \
        dvy = (lv[b * 3 + 1] + av[b * 3 + 2] * rB[0] - av[b * 3 + 0] * rB[2]) -                \
              (lv[a * 3 + 1] + av[a * 3 + 2] * rA[0] - av[a * 3 + 0] * rA[2]);                 \
        dvz = (lv[b * 3 + 2] + av[b * 3 + 0] * rB[1] - av[b * 3 + 1] * rB[0]) -                \
              (lv[a * 3 + 2] + av[a * 3 + 0] * rA[1] - av[a * 3 + 1] * rA[0]);                 \
    } while (0)

static int solve_contacts(OrWorld *w) {
    int K = w->n_contacts;
    if (K == 0) return 0;                          /* solver.py:197-198: cache kept */
    wake_sleepers(w);
    int n = w->n;
    double *invIw = (double *)malloc(sizeof(double) * 9 * (n ? n : 1));
    for (int i = 0; i < n; i++) {
        double R[9];
        or_quat_to_matrix(&w->q[i * 4], R);
        inv_inertia_world_einsum(R, &w->inv_inertia[i * 3], &invIw[i * 9]);
    }
    double *rest = (double *)malloc(sizeof(double) * K), *fric = (double *)malloc(sizeof(double) * K);
    double *nImp = (double *)calloc(K, sizeof(double)), *tImp = (double *)calloc(2 * K, sizeof(double));
    double *rA = (double *)malloc(sizeof(double) * 3 * K), *rB = (double *)malloc(sizeof(double) * 3 * K);
    double *t1 = (double *)malloc(sizeof(double) * 3 * K), *t2 = (double *)malloc(sizeof(double) * 3 * K);
    double *nM = (double *)malloc(sizeof(double) * K), *t1M = (double *)malloc(sizeof(double) * K);
    double *t2M = (double *)malloc(sizeof(double) * K), *vB = (double *)malloc(sizeof(double) * K);
    double *ima = (double *)malloc(sizeof(double) * K), *imb = (double *)malloc(sizeof(double) * K);
    for (int k = 0; k < K; k++) {                  /* solver.py:248-263 */
        int a = w->c_a[k], b = w->c_b[k];
        double fa, ra_, fb, rb_;
        int fca, rca, fcb, rcb;
        material(w, a, &fa, &ra_, &fca, &rca);
        material(w, b, &fb, &rb_, &fcb, &rcb);
        rest[k] = combine_val(ra_, rb_, rca);
        double mu;
        int ma = w->collider_material[a], mb = w->collider_material[b];
        if (pair_friction(w, ma, mb, &mu)) fric[k] = mu;
        else fric[k] = combine_val(fa, fb, fca);
        if (w->warm_start) {                       /* solver.py:222-233 */
            const double *p = &w->c_pt[k * 3];
            double best_d = 0.04;
            int best = -1;
            for (int c = 0; c < w->cache_n; c++) {
                if (w->cache_a[c] != a || w->cache_b[c] != b) continue;
                double d0 = p[0] - w->cache_pt[c * 3], d1 = p[1] - w->cache_pt[c * 3 + 1],
                       d2 = p[2] - w->cache_pt[c * 3 + 2];
                double d = d0 * d0 + d1 * d1 + d2 * d2;
                if (d < best_d) { best_d = d; best = c; }
            }
            if (best >= 0) {
                nImp[k] = w->cache_imp[best * 3];
                tImp[k * 2] = w->cache_imp[best * 3 + 1];
                tImp[k * 2 + 1] = w->cache_imp[best * 3 + 2];
            }
        }
    }
    double *lv = w->v, *av = w->w, *pos = w->pos;
    const double *point = w->c_pt, *normal = w->c_n;
    /* prepare (_solver_native.pyx:209-248) */
    for (int k = 0; k < K; k++) {
        int a = w->c_a[k], b = w->c_b[k];
        double imak = w->inv_mass[a], imbk = w->inv_mass[b];
        ima[k] = imak; imb[k] = imbk;
        for (int c = 0; c < 3; c++) {
            rA[k * 3 + c] = point[k * 3 + c] - pos[a * 3 + c];
            rB[k * 3 + c] = point[k * 3 + c] - pos[b * 3 + c];
        }
        double nx = normal[k * 3], ny = normal[k * 3 + 1], nz = normal[k * 3 + 2];
        double axx, ayy, azz;
        if ((nx >= 0 ? nx : -nx) < 0.9) { axx = 1.0; ayy = 0.0; azz = 0.0; }
        else { axx = 0.0; ayy = 1.0; azz = 0.0; }
        double t1x = ayy * nz - azz * ny, t1y = azz * nx - axx * nz, t1z = axx * ny - ayy * nx;
        double ln = sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
        double inv = ln > 1e-12 ? 1.0 / ln : 0.0;
        t1x *= inv; t1y *= inv; t1z *= inv;
        t1[k * 3] = t1x; t1[k * 3 + 1] = t1y; t1[k * 3 + 2] = t1z;
        t2[k * 3] = ny * t1z - nz * t1y;
        t2[k * 3 + 1] = nz * t1x - nx * t1z;
        t2[k * 3 + 2] = nx * t1y - ny * t1x;
        nM[k] = effmass(&rA[k * 3], &rB[k * 3], nx, ny, nz, invIw, a, b, imak, imbk);
        t1M[k] = effmass(&rA[k * 3], &rB[k * 3], t1x, t1y, t1z, invIw, a, b, imak, imbk);
        t2M[k] = effmass(&rA[k * 3], &rB[k * 3], t2[k * 3], t2[k * 3 + 1], t2[k * 3 + 2], invIw, a, b,
                         imak, imbk);
        double dvx, dvy, dvz;
        const double *ra = &rA[k * 3], *rb = &rB[k * 3];
        REL_VEL(lv, av, a, b, ra, rb, dvx, dvy, dvz);
        double vn0 = dvx * nx + dvy * ny + dvz * nz;
        vB[k] = vn0 < -w->restitution_threshold ? -rest[k] * vn0 : 0.0;
    }
    if (w->warm_start) {                           /* pyx:250-256 */
        for (int k = 0; k < K; k++) {
            int a = w->c_a[k], b = w->c_b[k];
            const double *nn = &normal[k * 3], *u = &t1[k * 3], *v = &t2[k * 3];
            apply_w(lv, av, a, b, ima[k], imb[k], invIw, &rA[k * 3], &rB[k * 3],
                    nImp[k] * nn[0] + tImp[k * 2] * u[0] + tImp[k * 2 + 1] * v[0],
                    nImp[k] * nn[1] + tImp[k * 2] * u[1] + tImp[k * 2 + 1] * v[1],
                    nImp[k] * nn[2] + tImp[k * 2] * u[2] + tImp[k * 2 + 1] * v[2]);
        }
    }
    for (int it = 0; it < w->velocity_iterations; it++) {   /* pyx:258-295 */
        for (int k = 0; k < K; k++) {
            int a = w->c_a[k], b = w->c_b[k];
            const double *ra = &rA[k * 3], *rb = &rB[k * 3];
            double nx = normal[k * 3], ny = normal[k * 3 + 1], nz = normal[k * 3 + 2];
            double dvx, dvy, dvz;
            REL_VEL(lv, av, a, b, ra, rb, dvx, dvy, dvz);
            double vn = dvx * nx + dvy * ny + dvz * nz;
            double nw = nImp[k] - nM[k] * (vn - vB[k]);
            if (nw < 0.0) nw = 0.0;
            double dL = nw - nImp[k];
            nImp[k] = nw;
            apply_w(lv, av, a, b, ima[k], imb[k], invIw, ra, rb, dL * nx, dL * ny, dL * nz);
            double maxf = fric[k] * nImp[k];
            REL_VEL(lv, av, a, b, ra, rb, dvx, dvy, dvz);
            const double *u = &t1[k * 3], *v = &t2[k * 3];
            double vt = dvx * u[0] + dvy * u[1] + dvz * u[2];
            double nt = tImp[k * 2] - t1M[k] * vt;
            if (nt > maxf) nt = maxf; else if (nt < -maxf) nt = -maxf;
            dL = nt - tImp[k * 2];
            tImp[k * 2] = nt;
            apply_w(lv, av, a, b, ima[k], imb[k], invIw, ra, rb, dL * u[0], dL * u[1], dL * u[2]);
            vt = dvx * v[0] + dvy * v[1] + dvz * v[2];
            nt = tImp[k * 2 + 1] - t2M[k] * vt;
            if (nt > maxf) nt = maxf; else if (nt < -maxf) nt = -maxf;
            dL = nt - tImp[k * 2 + 1];
            tImp[k * 2 + 1] = nt;
            apply_w(lv, av, a, b, ima[k], imb[k], invIw, ra, rb, dL * v[0], dL * v[1], dL * v[2]);
        }
    }
    for (int k = 0; k < K; k++) {                  /* pyx:298-312 */
        double vn = w->c_depth[k] - w->slop;
        if (vn <= 0.0) continue;
        double imak = ima[k], imbk = imb[k];
        if (imak + imbk <= 1e-12) continue;
        double dL = w->correction * vn / (imak + imbk);
        int a = w->c_a[k], b = w->c_b[k];
        for (int c = 0; c < 3; c++) {
            pos[a * 3 + c] -= imak * dL * normal[k * 3 + c];
            pos[b * 3 + c] += imbk * dL * normal[k * 3 + c];
        }
    }
    if (w->warm_start) {                           /* solver.py:271-278 */
        /* the impulses reach the contacts and the cache only with warm start on;
         * otherwise the contacts keep zeros and the cache its last contents */
        for (int k = 0; k < K; k++) {
            w->c_imp[k * 3] = nImp[k];
            w->c_imp[k * 3 + 1] = tImp[k * 2];
            w->c_imp[k * 3 + 2] = tImp[k * 2 + 1];
        }
        if (or_set_cache(w, K, w->c_a, w->c_b, w->c_pt, w->c_imp)) return -1;
    }
    free(invIw); free(rest); free(fric); free(nImp); free(tImp); free(rA); free(rB);
    free(t1); free(t2); free(nM); free(t1M); free(t2M); free(vB); free(ima); free(imb);
    return 0;
}

/* ------------------------------------------------------------------ */
/* joints (world.py:599-611, joints.py:60-212)                        */
/* ------------------------------------------------------------------ */
typedef struct {
    double invIa[9], invIb[9];
    double rA[3], rB[3], K[9], bias[3];
    double n[3], mass, bias_s;
} JointScratch;

static void inv_inertia_joint(const OrWorld *w, int i, double *W) {   /* joints.py:278-283 */
    if (i < 0) { for (int q = 0; q < 9; q++) W[q] = 0.0; return; }
    double R[9];
    or_quat_to_matrix(&w->q[i * 4], R);
    inv_inertia_world_gemm(R, &w->inv_inertia[i * 3], W);
}

static void mat3_mul_blas(const double *A, const double *B, double *C) {
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            double col[3] = {B[k], B[3 + k], B[6 + k]};
            C[i * 3 + k] = dot_blas(&A[i * 3], col);
        }
}

static void skew(const double *r, double *S) {   /* joints.py:16-19 */
    S[0] = 0.0; S[1] = -r[2]; S[2] = r[1];
    S[3] = r[2]; S[4] = 0.0; S[5] = -r[0];
    S[6] = -r[1]; S[7] = r[0]; S[8] = 0.0;
}

static void point_velocity(const OrWorld *w, int i, const double *r, double *out) {
    if (i < 0) { out[0] = out[1] = out[2] = 0.0; return; }
    double c[3];
    cross_np(&w->w[i * 3], r, c);
    for (int q = 0; q < 3; q++) out[q] = w->v[i * 3 + q] + c[q];
}

static void joint_apply(OrWorld *w, int i, const double *invI, const double *r, const double *P) {
    if (i < 0) return;
    double c[3];
    for (int q = 0; q < 3; q++) w->v[i * 3 + q] = w->v[i * 3 + q] + w->inv_mass[i] * P[q];
    cross_np(r, P, c);
    for (int q = 0; q < 3; q++) w->w[i * 3 + q] = w->w[i * 3 + q] + gemv_row(&invI[q * 3], c);
}

/* LU with partial pivoting for np.linalg.solve (joints.py:119) */
static void solve3(const double *Kin, const double *rhs, double *x) {
    double A[9], b[3];
    memcpy(A, Kin, sizeof(A));
    memcpy(b, rhs, sizeof(b));
    for (int j = 0; j < 3; j++) {
        int p = j;
        double best = fabs(A[j * 3 + j]);
        for (int i = j + 1; i < 3; i++)
            if (fabs(A[i * 3 + j]) > best) { best = fabs(A[i * 3 + j]); p = i; }
        if (p != j) {
            for (int k = 0; k < 3; k++) { double t = A[j * 3 + k]; A[j * 3 + k] = A[p * 3 + k]; A[p * 3 + k] = t; }
            double t = b[j]; b[j] = b[p]; b[p] = t;
        }
        for (int i = j + 1; i < 3; i++) {
            double l = A[i * 3 + j] / A[j * 3 + j];
            A[i * 3 + j] = l;
            for (int k = j + 1; k < 3; k++) A[i * 3 + k] = fma(-l, A[j * 3 + k], A[i * 3 + k]);
        }
    }
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < i; k++) b[i] = fma(-A[i * 3 + k], b[k], b[i]);
    for (int i = 2; i >= 0; i--) {
        for (int k = i + 1; k < 3; k++) b[i] = fma(-A[i * 3 + k], b[k], b[i]);
        b[i] = b[i] / A[i * 3 + i];
    }
    memcpy(x, b, sizeof(b));
}

static void joint_prepare(OrWorld *w, int j, JointScratch *s) {
    int t = w->j_type[j];
    if (t == OR_JOINT_MOTOR) {                   /* joints.py:198-202 */
        int body = w->j_a[j];
        inv_inertia_joint(w, body, s->invIa);
        const double *ax = &w->j_axis[j * 3];
        double u[3];
        for (int k = 0; k < 3; k++) {            /* axis @ invI (vec @ mat) */
            double col[3] = {s->invIa[k], s->invIa[3 + k], s->invIa[6 + k]};
            u[k] = dot_blas(ax, col);
        }
        double eff = dot_blas(u, ax);
        s->mass = eff > 1e-12 ? 1.0 / eff : 0.0;
        w->j_accum[j] = 0.0;
        return;
    }
    int a = w->j_a[j], b = w->j_b[j];
    inv_inertia_joint(w, a, s->invIa);
    inv_inertia_joint(w, b, s->invIb);
    if (t == OR_JOINT_POINT) {                   /* joints.py:86-102 */
        const double *anchor = &w->j_anchor[j * 3];
        int ids[2] = {a, b};
        double *locs[2] = {&w->j_local_a[j * 3], &w->j_local_b[j * 3]};
        uint8_t *has[2] = {&w->j_has_local_a[j], &w->j_has_local_b[j]};
        double *rs[2] = {s->rA, s->rB};
        double posv[2][3];
        for (int e = 0; e < 2; e++) {
            int i = ids[e];
            if (i >= 0 && !*has[e]) {            /* _to_local: R.T @ (pt - pos) */
                double R[9], d[3];
                or_quat_to_matrix(&w->q[i * 4], R);
                sub3(anchor, &w->pos[i * 3], d);
                for (int k = 0; k < 3; k++) {
                    double col[3] = {R[k], R[3 + k], R[6 + k]};
                    locs[e][k] = dot_blas(col, d);
                }
                *has[e] = 1;
            }
            double wa[3];
            if (i < 0) { for (int k = 0; k < 3; k++) { wa[k] = anchor[k]; posv[e][k] = anchor[k]; } }
            else {
                double R[9];
                or_quat_to_matrix(&w->q[i * 4], R);
                for (int k = 0; k < 3; k++) {
                    wa[k] = w->pos[i * 3 + k] + gemv_row(&R[k * 3], locs[e]);
                    posv[e][k] = w->pos[i * 3 + k];
                }
            }
            for (int k = 0; k < 3; k++) rs[e][k] = wa[k] - posv[e][k];
        }
        double im = (a < 0 ? 0.0 : w->inv_mass[a]) + (b < 0 ? 0.0 : w->inv_mass[b]);
        for (int q = 0; q < 9; q++) s->K[q] = (q % 4 == 0) ? im * 1.0 : im * 0.0;
        double S[9], T[9], M[9];
        skew(s->rA, S); mat3_mul_blas(S, s->invIa, T); mat3_mul_blas(T, S, M);
        for (int q = 0; q < 9; q++) s->K[q] = s->K[q] - M[q];
        skew(s->rB, S); mat3_mul_blas(S, s->invIb, T); mat3_mul_blas(T, S, M);
        for (int q = 0; q < 9; q++) s->K[q] = s->K[q] - M[q];
        for (int k = 0; k < 3; k++) {
            double pa = posv[0][k] + s->rA[k], pb = posv[1][k] + s->rB[k];
            s->bias[k] = 0.2 * (pb - pa);
        }
        return;
    }
    /* DistanceConstraint (joints.py:139-158) */
    const double *la = &w->j_anchor[j * 3], *lb = &w->j_anchor_b[j * 3];
    double pa[3], pb[3], d[3];
    for (int e = 0; e < 2; e++) {
        int i = e == 0 ? a : b;
        const double *loc = e == 0 ? la : lb;
        double *out = e == 0 ? pa : pb;
        if (i < 0) { for (int k = 0; k < 3; k++) out[k] = loc[k]; }
        else {
            double R[9];
            or_quat_to_matrix(&w->q[i * 4], R);
            for (int k = 0; k < 3; k++) out[k] = w->pos[i * 3 + k] + gemv_row(&R[k * 3], loc);
        }
    }
    sub3(pb, pa, d);
    double dist = norm_blas3(d);
    if (dist > 1e-9) { for (int k = 0; k < 3; k++) s->n[k] = d[k] / dist; }
    else { s->n[0] = 0.0; s->n[1] = 1.0; s->n[2] = 0.0; }
    if (!w->j_has_length[j]) { w->j_length[j] = dist; w->j_has_length[j] = 1; }
    for (int k = 0; k < 3; k++) {
        s->rA[k] = pa[k] - (a < 0 ? la[k] : w->pos[a * 3 + k]);
        s->rB[k] = pb[k] - (b < 0 ? la[k] : w->pos[b * 3 + k]);
    }
    double raxn[3], rbxn[3], u[3];
    cross_np(s->rA, s->n, raxn);
    cross_np(s->rB, s->n, rbxn);
    double k = (a < 0 ? 0.0 : w->inv_mass[a]) + (b < 0 ? 0.0 : w->inv_mass[b]);
    for (int q = 0; q < 3; q++) { double col[3] = {s->invIa[q], s->invIa[3 + q], s->invIa[6 + q]}; u[q] = dot_blas(raxn, col); }
    k += dot_blas(u, raxn);
    for (int q = 0; q < 3; q++) { double col[3] = {s->invIb[q], s->invIb[3 + q], s->invIb[6 + q]}; u[q] = dot_blas(rbxn, col); }
    k += dot_blas(u, rbxn);
    s->mass = k > 1e-12 ? 1.0 / k : 0.0;
    s->bias_s = 0.2 * (dist - w->j_length[j]);
}

static void joint_solve(OrWorld *w, int j, JointScratch *s, double dt) {
    int t = w->j_type[j];
    if (t == OR_JOINT_MOTOR) {                   /* joints.py:204-212 */
        int body = w->j_a[j];
        const double *ax = &w->j_axis[j * 3];
        double wv = dot_blas(&w->w[body * 3], ax);
        double impulse = s->mass * (w->j_target[j] - wv);
        double limit = w->j_max_force[j] * dt;
        double nw = w->j_accum[j] + impulse;
        if (nw < -limit) nw = -limit;
        if (nw > limit) nw = limit;
        impulse = nw - w->j_accum[j];
        w->j_accum[j] = nw;
        double P[3] = {ax[0] * impulse, ax[1] * impulse, ax[2] * impulse};
        for (int q = 0; q < 3; q++) w->w[body * 3 + q] = w->w[body * 3 + q] + gemv_row(&s->invIa[q * 3], P);
        return;
    }
    int a = w->j_a[j], b = w->j_b[j];
    double va[3], vb[3], P[3], nP[3];
    point_velocity(w, b, s->rB, vb);
    point_velocity(w, a, s->rA, va);
    if (t == OR_JOINT_POINT) {                   /* joints.py:114-121 */
        double rhs[3];
        for (int q = 0; q < 3; q++) rhs[q] = -((vb[q] - va[q]) + s->bias[q] / dt);
        solve3(s->K, rhs, P);
    } else {                                     /* joints.py:171-178 */
        double dv[3];
        sub3(vb, va, dv);
        double cdot = dot_blas(dv, s->n);
        double impulse = -s->mass * (cdot + s->bias_s / dt);
        for (int q = 0; q < 3; q++) P[q] = impulse * s->n[q];
    }
    neg3(P, nP);
    joint_apply(w, a, s->invIa, s->rA, nP);
    joint_apply(w, b, s->invIb, s->rB, P);
}

static int solve_joints(OrWorld *w) {
    int J = w->n_joints;
    if (J == 0) return 0;
    JointScratch *s = (JointScratch *)calloc(J, sizeof(JointScratch));
    if (!s) return -1;
    for (int j = 0; j < J; j++) {
        if (w->j_type[j] == OR_JOINT_MOTOR) { if (w->j_a[j] >= 0) wake(w, w->j_a[j]); }
        else {
            if (w->j_a[j] >= 0) wake(w, w->j_a[j]);
            if (w->j_b[j] >= 0) wake(w, w->j_b[j]);
        }
        joint_prepare(w, j, &s[j]);
    }
    for (int it = 0; it < w->joint_iterations; it++)
        for (int j = 0; j < J; j++) joint_solve(w, j, &s[j], w->dt);
    free(s);
    return 0;
}

/* ------------------------------------------------------------------ */
/* integration (backend.py:26-49, mathutil.py:32-41, 108-113)         */
/* ------------------------------------------------------------------ */
/* resolve_gravity with apply_volumes (world.py:386-396, gravity.py:82-108):
 * the world's vector, then every volume containing the body's position in
 * application order: replace sets, stop zeroes, otherwise the field adds */
static void body_gravity(const OrWorld *w, int i, double *g) {
    const double *pos = &w->pos[i * 3];
    for (int c = 0; c < 3; c++) g[c] = w->g[c];
    for (int k = 0; k < w->n_volumes; k++) {
        const int kind = w->vol_kind[k];
        const double *rc = &w->vol_rc[k * 3], *rr = &w->vol_rr[k * 3];
        int inside = 1;
        if (kind & OR_VOL_SPHERE) {                      /* gravity.py:22-25 */
            double d[3] = {pos[0] - rc[0], pos[1] - rc[1], pos[2] - rc[2]};
            inside = dot_blas(d, d) <= rr[0];
        } else if (kind & OR_VOL_BOX) {                  /* gravity.py:34-37 */
            for (int c = 0; c < 3; c++) inside &= fabs(pos[c] - rc[c]) <= rr[c];
        }
        if (!inside) continue;
        if (kind & OR_VOL_STOP) {
            g[0] = g[1] = g[2] = 0.0;
            continue;
        }
        double f[3];                                     /* field_at, gravity.py:66-79 */
        const double *fd = &w->vol_field[k * 3];
        if (kind & OR_VOL_POINT) {
            double d[3] = {fd[0] - pos[0], fd[1] - pos[1], fd[2] - pos[2]}, u[3];
            normalize3(d, u);
            for (int c = 0; c < 3; c++) f[c] = u[c] * w->vol_g[k];
        } else {
            for (int c = 0; c < 3; c++) f[c] = fd[c];
        }
        if (kind & OR_VOL_REPLACE) for (int c = 0; c < 3; c++) g[c] = f[c];
        else for (int c = 0; c < 3; c++) g[c] = g[c] + f[c];
    }
}

void or_integrate_forces(OrWorld *w) {
    double dt = w->dt;
    for (int i = 0; i < w->n; i++) {
        if (!(w->motion_type[i] == 2 && w->awake[i])) continue;
        double *v = &w->v[i * 3], *om = &w->w[i * 3];
        double gf = w->gravity_factor[i];
        double g[3];
        body_gravity(w, i, g);
        for (int c = 0; c < 3; c++) v[c] = v[c] + (g[c] * gf) * dt;
        double ld = w->lin_damp[i] + w->default_lin_damp;
        double ad = w->ang_damp[i] + w->default_ang_damp;
        double fl = 1.0 - ld * dt;
        fl = fl != fl ? fl : (fl > 0.0 ? fl : 0.0);
        for (int c = 0; c < 3; c++) v[c] = v[c] * fl;
        double speed = norm_axis3(v);
        double qd = w->quad_drag[i];
        double dv[3];
        for (int c = 0; c < 3; c++) dv[c] = ((qd * speed) * v[c]) * dt;
        for (int c = 0; c < 3; c++) v[c] = v[c] - dv[c];
        double fa = 1.0 - ad * dt;
        fa = fa != fa ? fa : (fa > 0.0 ? fa : 0.0);
        for (int c = 0; c < 3; c++) om[c] = om[c] * fa;
    }
}

void or_integrate_positions(OrWorld *w) {
    double dt = w->dt;
    for (int i = 0; i < w->n; i++) {
        int t = w->motion_type[i];
        if (!((t == 2 || t == 1) && w->awake[i])) continue;
        double *p = &w->pos[i * 3], *q = &w->q[i * 4];
        const double *v = &w->v[i * 3], *om = &w->w[i * 3];
        for (int c = 0; c < 3; c++) p[c] = p[c] + v[c] * dt;
        /* quat_mul((omega, 0), q) in the order of mathutil.py:36-41 */
        double ax = om[0], ay = om[1], az = om[2], aw = 0.0;
        double bx = q[0], by = q[1], bz = q[2], bw = q[3];
        double m[4];
        m[0] = aw * bx + ax * bw + ay * bz - az * by;
        m[1] = aw * by - ax * bz + ay * bw + az * bx;
        m[2] = aw * bz + ax * by - ay * bx + az * bw;
        m[3] = aw * bw - ax * bx - ay * by - az * bz;
        double s[4];
        for (int c = 0; c < 4; c++) s[c] = q[c] + (0.5 * m[c]) * dt;
        double n = sqrt(((s[0] * s[0] + s[1] * s[1]) + s[2] * s[2]) + s[3] * s[3]);
        double d = n > 1e-12 ? n : 1e-12;
        if (n != n) d = n;
        for (int c = 0; c < 4; c++) q[c] = s[c] / d;
    }
}

/* ------------------------------------------------------------------ */
/* sleeping (world.py:510-567)                                         */
/* ------------------------------------------------------------------ */
static int uf_find(int *parent, int x) {
    while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
    return x;
}

static void update_sleep(OrWorld *w) {
    int n = w->n;
    double dt = w->dt;
    double lin2 = 0.08 * 0.08, ang2 = 0.25 * 0.25;
    uint8_t *slow = (uint8_t *)calloc(n ? n : 1, 1), *ready = (uint8_t *)calloc(n ? n : 1, 1);
    uint8_t *contacted = (uint8_t *)calloc(n ? n : 1, 1), *to_sleep = (uint8_t *)calloc(n ? n : 1, 1);
    uint8_t *notready = (uint8_t *)calloc(n ? n : 1, 1);
    int *parent = (int *)malloc(sizeof(int) * (n ? n : 1));
    for (int i = 0; i < n; i++) {
        int dyn = w->motion_type[i] == 2;
        const double *v = &w->v[i * 3], *om = &w->w[i * 3];
        double s2 = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
        double a2 = (om[0] * om[0] + om[1] * om[1]) + om[2] * om[2];
        slow[i] = dyn && s2 < lin2 && a2 < ang2;
        if (slow[i]) w->sleep_timer[i] += dt; else w->sleep_timer[i] = 0.0;
        ready[i] = slow[i] && w->sleep_timer[i] > 0.4;
        parent[i] = i;
    }
    for (int k = 0; k < w->n_contacts; k++) {
        int a = w->c_a[k], b = w->c_b[k];
        int da = w->motion_type[a] == 2, db = w->motion_type[b] == 2;
        if (da) contacted[a] = 1;
        if (db) contacted[b] = 1;
        if (da && db) parent[uf_find(parent, a)] = uf_find(parent, b);
    }
    for (int i = 0; i < n; i++)
        if (contacted[i] && !ready[i]) notready[uf_find(parent, i)] = 1;
    for (int i = 0; i < n; i++) {
        w->island[i] = contacted[i] ? uf_find(parent, i) : -1;
        if (contacted[i]) { if (!notready[uf_find(parent, i)]) to_sleep[i] = 1; }
        else if (w->motion_type[i] == 2 && ready[i]) to_sleep[i] = 1;
    }
    for (int i = 0; i < n; i++) {
        int dyn = w->motion_type[i] == 2;
        if (to_sleep[i]) w->awake[i] = 0;
        if (dyn && !slow[i]) w->awake[i] = 1;
        if (!w->awake[i] && dyn) {
            for (int c = 0; c < 3; c++) { w->v[i * 3 + c] = 0.0; w->w[i * 3 + c] = 0.0; }
        }
    }
    free(slow); free(ready); free(contacted); free(to_sleep); free(notready); free(parent);
}

/* ------------------------------------------------------------------ */
/* the step (world.py:410-430)                                         */
/* ------------------------------------------------------------------ */
/* ------------------------------------------------------------------ */
/* trigger overlaps (triggers.py:24-72, world.py:662-676)              */
/* ------------------------------------------------------------------ */
/* collide.sphere_sphere is empty iff dist >= ra + rb (collide.py:56-66) */
static int py_sphere_sphere_hit(const Proxy *A, const Proxy *B) {
    double d[3] = {B->center[0] - A->center[0], B->center[1] - A->center[1], B->center[2] - A->center[2]};
    return !(norm_blas3(d) >= A->radius + B->radius);
}

/* collide.sphere_box is empty iff the clamped distance exceeds the radius
 * (collide.py:69-88); local = R.T @ (cs - cb), norm over the whole vector */
static int py_sphere_box_hit(const Proxy *S, const Proxy *B) {
    double v[3] = {S->center[0] - B->center[0], S->center[1] - B->center[1], S->center[2] - B->center[2]};
    double delta[3];
    for (int j = 0; j < 3; j++) {
        double col[3] = {B->R[j], B->R[3 + j], B->R[6 + j]};
        double l = dot_blas(col, v);
        double cl = l > -B->half[j] ? l : -B->half[j];
        cl = cl < B->half[j] ? cl : B->half[j];
        delta[j] = l - cl;
    }
    return !(norm_blas3(delta) > S->radius);
}

/* len(collide.collide(trg, other, PA, PB)) > 0 (collide.py:251-269): the
 * analytic routes for sphere/box pairs, GJK/EPA otherwise. box_box is
 * non-empty exactly when its separating-axis test finds no gap; that test is
 * taken from the compiled box_box here. */
static int shapes_overlap(OrWorld *w, int ts, int trg, int os, int other, double *sa, double *sb) {
    Proxy A, B;
    make_proxy_shape(w, ts, trg, &A, sa);
    make_proxy_shape(w, os, other, &B, sb);
    const int ka = A.kind, kb = B.kind;
    if (ka == OR_SHAPE_SPHERE && kb == OR_SHAPE_SPHERE) return py_sphere_sphere_hit(&A, &B);
    if (ka == OR_SHAPE_SPHERE && kb == OR_SHAPE_BOX) return py_sphere_box_hit(&A, &B);
    if (ka == OR_SHAPE_BOX && kb == OR_SHAPE_SPHERE) return py_sphere_box_hit(&B, &A);
    double nrm[3], pts[12], dep[4];
    if (ka == OR_SHAPE_BOX && kb == OR_SHAPE_BOX)
        return or_box_box(A.center, A.R, A.half, B.center, B.R, B.half, nrm, pts, dep) > 0;
    return collide_convex(&A, &B, nrm, pts, dep) > 0;
}

/* this step's (trigger, other) overlaps in pair order: a pair with a sensor
 * on either body (the first body's when both have one) against the other
 * body's collider, else its sensor (triggers.py:46-72) */
static int trigger_overlaps(OrWorld *w) {
    Caps *cp = caps_for(w);
    w->n_overlaps = 0;
    if (!w->trigger_shape) return 0;
    int maxpts = 1;
    for (int s = 0; s < w->n_shapes; s++)
        if (w->shape_type[s] == OR_SHAPE_CONVEX && w->shape_pt_cnt[s] > maxpts) maxpts = w->shape_pt_cnt[s];
    double *sa = (double *)malloc(sizeof(double) * 3 * maxpts);
    double *sb = (double *)malloc(sizeof(double) * 3 * maxpts);
    int rc = 0;
    for (int p = 0; p < w->n_pairs; p++) {
        const int i = w->pairs[p * 2], j = w->pairs[p * 2 + 1];
        const int ti = trigger_of(w, i), tj = trigger_of(w, j);
        if (ti < 0 && tj < 0) continue;
        const int trg = ti >= 0 ? i : j, other = ti >= 0 ? j : i;
        const int ts = ti >= 0 ? ti : tj;
        int os = w->collider_shape[other];
        if (os < 0) os = trigger_of(w, other);
        if (os < 0) continue;
        if (!shapes_overlap(w, ts, trg, os, other, sa, sb)) continue;
        const int k = w->n_overlaps;
        int32_t cap = cp->overlap_cap;
        w->ov_trg = (int32_t *)grow(w->ov_trg, sizeof(int32_t), k + 1, &cap);
        cap = cp->overlap_cap;
        w->ov_other = (int32_t *)grow(w->ov_other, sizeof(int32_t), k + 1, &cap);
        cp->overlap_cap = cap;
        if (!w->ov_trg || !w->ov_other) { rc = -1; break; }
        w->ov_trg[k] = trg;
        w->ov_other[k] = other;
        w->n_overlaps = k + 1;
    }
    free(sa); free(sb);
    return rc;
}

int or_step(OrWorld *w) {
    int n = w->n;
    memcpy(w->prev_pos, w->pos, sizeof(double) * 3 * n);
    memcpy(w->prev_q, w->q, sizeof(double) * 4 * n);
    or_integrate_forces(w);
    w->n_pairs = w->n_solid = w->n_contacts = 0;
    if (w->has_collision) {
        or_refit(w);
        if (or_broadphase(w)) return -1;
        if (narrowphase(w)) return -2;
        if (solve_contacts(w)) return -3;
        if (trigger_overlaps(w)) return -5;
    }
    if (w->n_joints) { if (solve_joints(w)) return -4; }
    or_integrate_positions(w);
    if (w->sleep_enabled) update_sleep(w);
    else for (int i = 0; i < n; i++) w->island[i] = -1;
    return 0;
}

int or_set_cache(OrWorld *w, int32_t n, const int32_t *a, const int32_t *b, const double *pt,
                 const double *imp) {
    Caps *cp = caps_for(w);
    int32_t cap = cp->cache_cap;
    int32_t *na = (int32_t *)malloc(sizeof(int32_t) * (n ? n : 1));
    int32_t *nb = (int32_t *)malloc(sizeof(int32_t) * (n ? n : 1));
    double *np_ = (double *)malloc(sizeof(double) * 3 * (n ? n : 1));
    double *ni = (double *)malloc(sizeof(double) * 3 * (n ? n : 1));
    if (!na || !nb || !np_ || !ni) return -1;
    memcpy(na, a, sizeof(int32_t) * n); memcpy(nb, b, sizeof(int32_t) * n);
    memcpy(np_, pt, sizeof(double) * 3 * n); memcpy(ni, imp, sizeof(double) * 3 * n);
    free(w->cache_a); free(w->cache_b); free(w->cache_pt); free(w->cache_imp);
    w->cache_a = na; w->cache_b = nb; w->cache_pt = np_; w->cache_imp = ni;
    w->cache_n = n;
    cp->cache_cap = n > cap ? n : cap;
    return 0;
}

void or_free(OrWorld *w) {
    free(w->pairs); free(w->solid); free(w->c_a); free(w->c_b); free(w->c_pt); free(w->c_n);
    free(w->c_depth); free(w->c_imp); free(w->cache_a); free(w->cache_b); free(w->cache_pt);
    free(w->cache_imp); free(w->ov_trg); free(w->ov_other);
    w->ov_trg = w->ov_other = NULL;
    w->n_overlaps = 0;
    w->pairs = w->solid = w->c_a = w->c_b = w->cache_a = w->cache_b = NULL;
    w->c_pt = w->c_n = w->c_depth = w->c_imp = w->cache_pt = w->cache_imp = NULL;
    w->n_pairs = w->n_solid = w->n_contacts = w->cache_n = 0;
    CapEntry **pp = &g_caps;
    while (*pp) {
        if ((*pp)->w == w) { CapEntry *e = *pp; *pp = e->next; free(e); break; }
        pp = &(*pp)->next;
    }
    (void)g_mat_w;
}

/* ------------------------------------------------------------------ */
/* capsule against a batch of triangles (_collide_native.pyx:347-574, */
/* the compiled form of collide.py:309-382)                            */
/* ------------------------------------------------------------------ */
static inline double dot3_seq(const double *a, const double *b) {
    /* _dot3 (_collide_native.pyx:16-17): left to right */
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* closest point on triangle abc to p, Ericson's Voronoi regions in the
 * order _closest_on_tri tests them (_collide_native.pyx:364-410) */
static void tri_closest(const double *p, const double *a, const double *b, const double *c,
                        double *out) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int m = 0; m < 3; m++) { ab[m] = b[m] - a[m]; ac[m] = c[m] - a[m]; ap[m] = p[m] - a[m]; }
    const double d1 = dot3_seq(ab, ap), d2 = dot3_seq(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { for (int m = 0; m < 3; m++) out[m] = a[m]; return; }
    for (int m = 0; m < 3; m++) bp[m] = p[m] - b[m];
    const double d3 = dot3_seq(ab, bp), d4 = dot3_seq(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { for (int m = 0; m < 3; m++) out[m] = b[m]; return; }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double v = d1 / (d1 - d3);
        for (int m = 0; m < 3; m++) out[m] = a[m] + v * ab[m];
        return;
    }
    for (int m = 0; m < 3; m++) cp[m] = p[m] - c[m];
    const double d5 = dot3_seq(ab, cp), d6 = dot3_seq(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { for (int m = 0; m < 3; m++) out[m] = c[m]; return; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double w = d2 / (d2 - d6);
        for (int m = 0; m < 3; m++) out[m] = a[m] + w * ac[m];
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int m = 0; m < 3; m++) out[m] = b[m] + w * (c[m] - b[m]);
        return;
    }
    const double inv = 1.0 / (va + vb + vc);
    const double v = vb * inv, w = vc * inv;
    for (int m = 0; m < 3; m++) out[m] = a[m] + ab[m] * v + ac[m] * w;
}

static inline double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

/* closest points of segments p1q1 and p2q2 (_collide_native.pyx:413-451) */
static void seg_closest(const double *p1, const double *q1, const double *p2, const double *q2,
                        double *o1, double *o2) {
    double d1[3], d2[3], r[3], s, t;
    for (int m = 0; m < 3; m++) { d1[m] = q1[m] - p1[m]; d2[m] = q2[m] - p2[m]; r[m] = p1[m] - p2[m]; }
    const double aa = dot3_seq(d1, d1), e = dot3_seq(d2, d2), f = dot3_seq(d2, r);
    if (aa <= EPS_COLLIDE && e <= EPS_COLLIDE) {
        for (int m = 0; m < 3; m++) { o1[m] = p1[m]; o2[m] = p2[m]; }
        return;
    }
    if (aa <= EPS_COLLIDE) {
        s = 0.0;
        t = clamp01(f / e);
    } else {
        const double cc = dot3_seq(d1, r);
        if (e <= EPS_COLLIDE) {
            t = 0.0;
            s = clamp01(-cc / aa);
        } else {
            const double bb = dot3_seq(d1, d2);
            const double den = aa * e - bb * bb;
            s = den > EPS_COLLIDE ? clamp01((bb * f - cc * e) / den) : 0.0;
            t = (bb * s + f) / e;
            if (t < 0.0) {
                t = 0.0;
                s = clamp01(-cc / aa);
            } else if (t > 1.0) {
                t = 1.0;
                s = clamp01((bb - cc) / aa);
            }
        }
    }
    for (int m = 0; m < 3; m++) { o1[m] = p1[m] + d1[m] * s; o2[m] = p2[m] + d2[m] * t; }
}

/* one triangle; returns 1 on contact (point on the triangle, normal from the
 * triangle toward the capsule, depth) */
static int capsule_triangle_one(const double *c0, const double *c1, const double *centre, double radius,
                                const double *v0, const double *v1, const double *v2,
                                double *point, double *normal, double *depth) {
    double e1[3], e2[3], face[3], fn[3], tp[3];
    const double *ends[2] = {c0, c1};
    for (int m = 0; m < 3; m++) { e1[m] = v1[m] - v0[m]; e2[m] = v2[m] - v0[m]; }
    face[0] = e1[1] * e2[2] - e1[2] * e2[1];
    face[1] = e1[2] * e2[0] - e1[0] * e2[2];
    face[2] = e1[0] * e2[1] - e1[1] * e2[0];
    const double face_len = sqrt(dot3_seq(face, face));
    /* over the face: pushed back to the side the capsule's centre is on,
     * by the deepest cap end whose foot lies on the triangle */
    if (face_len > EPS_COLLIDE) {
        for (int m = 0; m < 3; m++) fn[m] = face[m] / face_len;
        double g[3] = {centre[0] - v0[0], centre[1] - v0[1], centre[2] - v0[2]};
        if (fn[0] * g[0] + fn[1] * g[1] + fn[2] * g[2] < 0.0)
            for (int m = 0; m < 3; m++) fn[m] = -fn[m];
        int found = 0;
        double best = -1e300, bp[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < 2; k++) {
            const double *sp = ends[k];
            for (int m = 0; m < 3; m++) g[m] = sp[m] - v0[m];
            const double h = fn[0] * g[0] + fn[1] * g[1] + fn[2] * g[2];
            double foot[3];
            for (int m = 0; m < 3; m++) foot[m] = sp[m] - fn[m] * h;
            tri_closest(sp, v0, v1, v2, tp);
            for (int m = 0; m < 3; m++) g[m] = foot[m] - tp[m];
            if (g[0] * g[0] + g[1] * g[1] + g[2] * g[2] > EPS_COLLIDE * EPS_COLLIDE) continue;
            const double reach = radius - h;
            if (reach > 0.0 && reach > best) {
                best = reach;
                found = 1;
                for (int m = 0; m < 3; m++) bp[m] = tp[m];
            }
        }
        if (found) {
            *depth = best;
            for (int m = 0; m < 3; m++) { point[m] = bp[m]; normal[m] = fn[m]; }
            return 1;
        }
    }
    /* off the rim: nearest of the cap ends to the triangle and of the axis
     * to the three edges, first strict minimum */
    double best_d2 = 1e300, bsp[3] = {0.0, 0.0, 0.0}, btp[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 2; k++) {
        const double *sp = ends[k];
        tri_closest(sp, v0, v1, v2, tp);
        const double gx = sp[0] - tp[0], gy = sp[1] - tp[1], gz = sp[2] - tp[2];
        const double d2 = gx * gx + gy * gy + gz * gz;
        if (d2 < best_d2) {
            best_d2 = d2;
            for (int m = 0; m < 3; m++) { bsp[m] = sp[m]; btp[m] = tp[m]; }
        }
    }
    const double *ea[3] = {v0, v1, v2}, *eb[3] = {v1, v2, v0};
    for (int k = 0; k < 3; k++) {
        double ax[3], ed[3];
        seg_closest(c0, c1, ea[k], eb[k], ax, ed);
        const double gx = ax[0] - ed[0], gy = ax[1] - ed[1], gz = ax[2] - ed[2];
        const double d2 = gx * gx + gy * gy + gz * gz;
        if (d2 < best_d2) {
            best_d2 = d2;
            for (int m = 0; m < 3; m++) { bsp[m] = ax[m]; btp[m] = ed[m]; }
        }
    }
    if (best_d2 >= radius * radius) return 0;
    const double dist = sqrt(best_d2);
    if (dist > EPS_COLLIDE) {
        for (int m = 0; m < 3; m++) normal[m] = (bsp[m] - btp[m]) / dist;
    } else if (face_len > EPS_COLLIDE) {
        for (int m = 0; m < 3; m++) normal[m] = face[m] / face_len;
    } else {
        normal[0] = normal[1] = normal[2] = 0.0;
    }
    *depth = radius - dist;
    for (int m = 0; m < 3; m++) point[m] = btp[m];
    return 1;
}

void or_capsule_triangles(const double *p0, const double *p1, double radius, const double *verts,
                          int64_t n, uint8_t *hit, double *points, double *normals, double *depths) {
    double centre[3];
    for (int m = 0; m < 3; m++) centre[m] = (p0[m] + p1[m]) * 0.5;
    for (int64_t i = 0; i < n; i++) {
        const double *t = &verts[i * 9];
        hit[i] = (uint8_t)capsule_triangle_one(p0, p1, centre, radius, t, t + 3, t + 6, &points[i * 3],
                                               &normals[i * 3], &depths[i]);
    }
}

/* ------------------------------------------------------------------ */
/* triangle meshes: the uniform grid (trigrid.py:63-218) and the mesh  */
/* route of collide.collide (collide.py:272-306)                       */
/* ------------------------------------------------------------------ */
typedef struct {
    int T, exact;                 /* exact: fewer than 256 triangles, no grid */
    const double *lo, *hi;        /* T*3 triangle bounds */
    double glo[3], ghi[3], cell;
    int shape[3];
    int *cell_off, *cell_tri;     /* CSR over dense cell ids (i*s1 + j)*s2 + k */
    int *big, nbig;
} TriGrid;

/* numpy / CPython float floor division (npy_divmod): fmod, then snap */
static double py_floordiv(double a, double b) {
    double mod = fmod(a, b);
    double div = (a - mod) / b;
    if (mod != 0.0) {
        if ((b < 0) != (mod < 0)) { mod += b; div -= 1.0; }
    }
    double fd;
    if (div != 0.0) {
        fd = floor(div);
        if (div - fd > 0.5) fd += 1.0;
    } else {
        fd = copysign(0.0, a / b);
    }
    return fd;
}

/* np.floor((p - low) / cell).astype(int), clipped to [0, cap] */
static int64_t grid_cell_of(double p, double low, double cell, int64_t cap) {
    int64_t r = (int64_t)floor((p - low) / cell);
    return r < 0 ? 0 : (r > cap ? cap : r);
}

static void grid_build(TriGrid *g, int T, const double *lo, const double *hi) {
    memset(g, 0, sizeof(*g));
    g->T = T; g->lo = lo; g->hi = hi;
    if (T < 256) { g->exact = 1; return; }              /* SMALLEST_WORTH_BINNING */
    for (int c = 0; c < 3; c++) {
        double mn = lo[c], mx = hi[c];
        for (int t = 1; t < T; t++) {
            if (lo[t * 3 + c] < mn) mn = lo[t * 3 + c];
            if (hi[t * 3 + c] > mx) mx = hi[t * 3 + c];
        }
        g->glo[c] = mn; g->ghi[c] = mx;
    }
    double ext = 0.0;
    for (int c = 0; c < 3; c++) {
        double e = g->ghi[c] - g->glo[c];
        e = e > 1e-9 ? e : 1e-9;
        if (c == 0 || e > ext) ext = e;
    }
    g->cell = ext / 64.0;                                 /* TARGET_CELLS */
    const int64_t cap = ((int64_t)1 << 30) - 1;
    int64_t *first = (int64_t *)malloc(sizeof(int64_t) * 3 * T), *last = (int64_t *)malloc(sizeof(int64_t) * 3 * T);
    int64_t smax[3] = {0, 0, 0};
    for (int t = 0; t < T; t++)
        for (int c = 0; c < 3; c++) {
            first[t * 3 + c] = grid_cell_of(lo[t * 3 + c], g->glo[c], g->cell, cap);
            last[t * 3 + c] = grid_cell_of(hi[t * 3 + c], g->glo[c], g->cell, cap);
            if (last[t * 3 + c] > smax[c]) smax[c] = last[t * 3 + c];
        }
    for (int c = 0; c < 3; c++) g->shape[c] = (int)(smax[c] + 1);
    const int64_t ncell = (int64_t)g->shape[0] * g->shape[1] * g->shape[2];
    g->cell_off = (int *)calloc((size_t)ncell + 1, sizeof(int));
    g->big = (int *)malloc(sizeof(int) * (T ? T : 1));
    for (int pass = 0; pass < 2; pass++) {
        int64_t fill_base = 0;
        (void)fill_base;
        for (int t = 0; t < T; t++) {
            const int64_t *f = &first[t * 3], *l = &last[t * 3];
            const int64_t span = (l[0] - f[0] + 1) * (l[1] - f[1] + 1) * (l[2] - f[2] + 1);
            if (span > 64) {                              /* BIG_CELL_LIMIT */
                if (pass == 0) g->big[g->nbig++] = t;
                continue;
            }
            for (int64_t i = f[0]; i <= l[0]; i++)
                for (int64_t j = f[1]; j <= l[1]; j++)
                    for (int64_t k = f[2]; k <= l[2]; k++) {
                        const int64_t id = (i * g->shape[1] + j) * g->shape[2] + k;
                        if (pass == 0) g->cell_off[id + 1]++;
                        else g->cell_tri[g->cell_off[id]++] = t;
                    }
        }
        if (pass == 0) {
            for (int64_t id = 0; id < ncell; id++) g->cell_off[id + 1] += g->cell_off[id];
            g->cell_tri = (int *)malloc(sizeof(int) * (g->cell_off[ncell] ? g->cell_off[ncell] : 1));
        } else {
            for (int64_t id = ncell; id > 0; id--) g->cell_off[id] = g->cell_off[id - 1];
            g->cell_off[0] = 0;
        }
    }
    free(first); free(last);
}

static void grid_free(TriGrid *g) { free(g->cell_off); free(g->cell_tri); free(g->big); }

static int cmp_int(const void *x, const void *y) { int a = *(const int *)x, b = *(const int *)y; return (a > b) - (a < b); }

/* TriangleGrid.box (trigrid.py:99-111, 183-218): candidate triangles of
 * [low, high], ascending, no repeats; returns the count, *out malloc'd */
static int grid_box(const TriGrid *g, const double *low, const double *high, int **out) {
    int n = 0, cap = 64;
    int *c = (int *)malloc(sizeof(int) * cap);
    if (g->exact) {
        for (int t = 0; t < g->T; t++) {
            int keep = 1;
            for (int k = 0; k < 3; k++) keep &= g->lo[t * 3 + k] <= high[k] && g->hi[t * 3 + k] >= low[k];
            if (!keep) continue;
            if (n == cap) { cap *= 2; c = (int *)realloc(c, sizeof(int) * cap); }
            c[n++] = t;
        }
        *out = c;
        return n;
    }
    int outside = 0;
    for (int k = 0; k < 3; k++) outside |= low[k] > g->ghi[k] || high[k] < g->glo[k];
    if (!outside) {
        int f[3], l[3];
        for (int k = 0; k < 3; k++) {
            double a = py_floordiv(low[k] - g->glo[k], g->cell), b = py_floordiv(high[k] - g->glo[k], g->cell);
            int64_t ia = (int64_t)a, ib = (int64_t)b;
            ia = ia < 0 ? 0 : ia; ib = ib < 0 ? 0 : ib;
            f[k] = (int)(ia > g->shape[k] - 1 ? g->shape[k] - 1 : ia);
            l[k] = (int)(ib > g->shape[k] - 1 ? g->shape[k] - 1 : ib);
        }
        for (int i = f[0]; i <= l[0]; i++)
            for (int j = f[1]; j <= l[1]; j++)
                for (int k = f[2]; k <= l[2]; k++) {
                    const int64_t id = ((int64_t)i * g->shape[1] + j) * g->shape[2] + k;
                    for (int q = g->cell_off[id]; q < g->cell_off[id + 1]; q++) {
                        if (n == cap) { cap *= 2; c = (int *)realloc(c, sizeof(int) * cap); }
                        c[n++] = g->cell_tri[q];
                    }
                }
    }
    for (int q = 0; q < g->nbig; q++) {
        if (n == cap) { cap *= 2; c = (int *)realloc(c, sizeof(int) * cap); }
        c[n++] = g->big[q];
    }
    qsort(c, n, sizeof(int), cmp_int);
    int m = 0;
    for (int q = 0; q < n; q++) if (m == 0 || c[q] != c[m - 1]) c[m++] = c[q];
    *out = c;
    return m;
}

/* world AABB of a support proxy (body.py: aabb of each proxy), no margin */
static void proxy_aabb(const OrWorld *w, int si, int i, const Proxy *P, double *lo, double *hi) {
    const double *pos = &w->pos[i * 3];
    if (P->kind == OR_SHAPE_SPHERE) {
        for (int c = 0; c < 3; c++) { lo[c] = pos[c] - P->radius; hi[c] = pos[c] + P->radius; }
    } else if (P->kind == OR_SHAPE_BOX) {                 /* _box_corners(half) @ R.T + center */
        for (int c = 0; c < 3; c++) { lo[c] = INFINITY; hi[c] = -INFINITY; }
        for (int k = 0; k < 8; k++) {
            double s[3] = {(k & 1) ? P->half[0] : -P->half[0], (k & 2) ? P->half[1] : -P->half[1],
                           (k & 4) ? P->half[2] : -P->half[2]};
            for (int c = 0; c < 3; c++) {
                double x = dot_blas(s, &P->R[c * 3]) + P->center[c];   /* numpy's dgemm order, probed */
                if (x < lo[c]) lo[c] = x;
                if (x > hi[c]) hi[c] = x;
            }
        }
    } else if (P->kind == OR_SHAPE_CAPSULE) {
        for (int c = 0; c < 3; c++) {
            lo[c] = (P->p0[c] < P->p1[c] ? P->p0[c] : P->p1[c]) - P->radius;
            hi[c] = (P->p0[c] > P->p1[c] ? P->p0[c] : P->p1[c]) + P->radius;
        }
    } else {
        for (int c = 0; c < 3; c++) {
            double mn = P->world[c], mx = P->world[c];
            for (int q = 1; q < P->m; q++) {
                double x = P->world[q * 3 + c];
                if (x < mn) mn = x;
                if (x > mx) mx = x;
            }
            lo[c] = mn; hi[c] = mx;
        }
    }
    (void)si;
}

/* the mesh route (collide.py:272-306): a capsule against every candidate
 * triangle at once (capsule_triangle_batch), any other proxy through GJK/EPA
 * one candidate triangle at a time; contacts in candidate order, normals
 * from a to b */
/* A mesh body's world points, triangle bounds and grid, built once per
 * narrowphase pass (the reference caches the proxy per step, narrowphase.py:40-48) */
typedef struct { const OrWorld *w; int body, pass; double *wp, *tlo, *thi; TriGrid g; } MeshCache;
#define MESH_CACHE 8
static MeshCache g_mesh_cache[MESH_CACHE];
static int g_mesh_next = 0;

static MeshCache *mesh_body_tables(OrWorld *w, int mb) {
    for (int k = 0; k < MESH_CACHE; k++) {
        MeshCache *m = &g_mesh_cache[k];
        if (m->w == w && m->body == mb && m->pass == g_mesh_pass && m->wp) return m;
    }
    MeshCache *m = &g_mesh_cache[g_mesh_next];
    g_mesh_next = (g_mesh_next + 1) % MESH_CACHE;
    if (m->wp) { free(m->wp); free(m->tlo); free(m->thi); grid_free(&m->g); }
    const int ms = w->collider_shape[mb];
    double R[9];
    or_quat_to_matrix(&w->q[mb * 4], R);
    const int np_ = w->shape_pt_cnt[ms], T = w->shape_tri_cnt[ms];
    m->wp = (double *)malloc(sizeof(double) * 3 * (np_ ? np_ : 1));
    convex_world_points(w, ms, &w->pos[mb * 3], R, m->wp);
    m->tlo = (double *)malloc(sizeof(double) * 3 * (T ? T : 1));
    m->thi = (double *)malloc(sizeof(double) * 3 * (T ? T : 1));
    const int32_t *tri = &w->tris[(size_t)w->shape_tri_off[ms] * 3];
    for (int t = 0; t < T; t++)
        for (int c = 0; c < 3; c++) {
            double x0 = m->wp[tri[t * 3] * 3 + c], x1 = m->wp[tri[t * 3 + 1] * 3 + c], x2 = m->wp[tri[t * 3 + 2] * 3 + c];
            double mn = x0 < x1 ? x0 : x1, mx = x0 > x1 ? x0 : x1;
            m->tlo[t * 3 + c] = mn < x2 ? mn : x2;
            m->thi[t * 3 + c] = mx > x2 ? mx : x2;
        }
    grid_build(&m->g, T, m->tlo, m->thi);
    m->w = w; m->body = mb; m->pass = g_mesh_pass;
    return m;
}

static int collide_mesh(OrWorld *w, Caps *cp, int a, int b) {
    const int mesh_is_a = w->shape_type[w->collider_shape[a]] == OR_SHAPE_TRIMESH;
    const int mb = mesh_is_a ? a : b, ob = mesh_is_a ? b : a;
    const int ms = w->collider_shape[mb], os = w->collider_shape[ob];
    MeshCache *mc = mesh_body_tables(w, mb);
    const double *wp = mc->wp;
    const int32_t *tri = &w->tris[(size_t)w->shape_tri_off[ms] * 3];
    const TriGrid g = mc->g;
    int omax = w->shape_type[os] == OR_SHAPE_CONVEX ? w->shape_pt_cnt[os] : 1;
    double *so = (double *)malloc(sizeof(double) * 3 * (omax > 0 ? omax : 1));
    Proxy O;
    make_proxy_shape(w, os, ob, &O, so);
    double lo[3], hi[3];
    proxy_aabb(w, os, ob, &O, lo, hi);
    int *cand = NULL;
    const int nc = grid_box(&g, lo, hi, &cand);
    int rc = 0;
    for (int q = 0; q < nc && !rc; q++) {
        const int t = cand[q];
        const double *v0 = &wp[tri[t * 3] * 3], *v1 = &wp[tri[t * 3 + 1] * 3], *v2 = &wp[tri[t * 3 + 2] * 3];
        double pt[3], nrm[3], dep;
        int hit;
        if (O.kind == OR_SHAPE_CAPSULE) {
            double centre[3];
            for (int c = 0; c < 3; c++) centre[c] = (O.p0[c] + O.p1[c]) * 0.5;
            hit = capsule_triangle_one(O.p0, O.p1, centre, O.radius, v0, v1, v2, pt, nrm, &dep);
            if (hit && !mesh_is_a) for (int c = 0; c < 3; c++) nrm[c] = -nrm[c];
        } else {
            /* TriangleProxy (body.py:135-152): a three-point convex */
            double tv[9];
            for (int c = 0; c < 3; c++) { tv[c] = v0[c]; tv[3 + c] = v1[c]; tv[6 + c] = v2[c]; }
            Proxy P;
            memset(&P, 0, sizeof(P));
            P.kind = OR_SHAPE_CONVEX; P.world = tv; P.m = 3;
            double pts[12], deps[4];
            hit = mesh_is_a ? collide_convex(&P, &O, nrm, pts, deps) : collide_convex(&O, &P, nrm, pts, deps);
            if (hit > 0) { for (int c = 0; c < 3; c++) pt[c] = pts[c]; dep = deps[0]; }
            hit = hit > 0;
        }
        if (hit) rc = push_contact(w, cp, a, b, pt, nrm, dep);
    }
    free(cand); free(so);
    return rc;
}
