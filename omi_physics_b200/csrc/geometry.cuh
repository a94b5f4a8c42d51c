// Device geometry for the step, float64.
//
// This translation unit is compiled with --fmad=false: every a*b+c below is a
// separately rounded multiply and add, as in the reference's Cython C code
// (_collide_native.pyx, _solver_native.pyx) and numpy's elementwise ops. The
// only fused operations are the explicit fma() calls, placed exactly where
// numpy routes a 3-vector product through BLAS (np.dot, matmul, vec@mat: the
// chain fma(a2,b2, fma(a1,b1, a0*b0)); matrix@vector: fma(a2,b2, fma(a0,b0,
// a1*b1))). That keeps the GPU result bit-identical to the reference.
#pragma once
#include <cmath>
#include <cstdint>

namespace omi {

constexpr double EPS_COLLIDE = 1e-9;   // _collide_native.pyx:13
constexpr double EPS_GJK = 1e-10;      // gjk.py:19

__device__ __forceinline__ double dot_blas(const double *a, const double *b) {
    return fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0]));
}
__device__ __forceinline__ double gemv_row(const double *r, const double *x) {
    return fma(r[2], x[2], fma(r[0], x[0], r[1] * x[1]));
}
__device__ __forceinline__ void cross_np(const double *a, const double *b, double *c) {
    double x = a[1] * b[2] - a[2] * b[1];
    double y = a[2] * b[0] - a[0] * b[2];
    double z = a[0] * b[1] - a[1] * b[0];
    c[0] = x; c[1] = y; c[2] = z;
}
__device__ __forceinline__ void sub3(const double *a, const double *b, double *c) {
    c[0] = a[0] - b[0]; c[1] = a[1] - b[1]; c[2] = a[2] - b[2];
}
__device__ __forceinline__ void neg3(const double *a, double *c) {
    c[0] = -a[0]; c[1] = -a[1]; c[2] = -a[2];
}
// np.maximum(x, floor) for the positive floors used here (NaN propagates)
__device__ __forceinline__ double np_max(double x, double floor) {
    return (x != x) ? x : (x > floor ? x : floor);
}
// mathutil.normalize on a 3-vector (mathutil.py:21): norm over axis, no BLAS
__device__ __forceinline__ void normalize3(const double *v, double *o) {
    double n = sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
    double d = np_max(n, 1e-12);
    o[0] = v[0] / d; o[1] = v[1] / d; o[2] = v[2] / d;
}

// CapsuleProxy segment ends (body.py:84-91): axis = R @ (0, 1, 0) as one
// dgemv row each, p0 = c - axis * hh, p1 = c + axis * hh
__device__ __forceinline__ void capsule_ends(const double *c, const double *R, double hh, double *p0,
                                             double *p1) {
    const double y[3] = {0.0, 1.0, 0.0};
    for (int k = 0; k < 3; k++) {
        const double a = gemv_row(&R[k * 3], y) * hh;
        p0[k] = c[k] - a;
        p1[k] = c[k] + a;
    }
}

// mathutil.quat_to_matrix (mathutil.py:59-76); R row-major, columns = axes
__device__ __forceinline__ void quat_to_matrix(const double *qi, double *m) {
    double n = sqrt(((qi[0] * qi[0] + qi[1] * qi[1]) + qi[2] * qi[2]) + qi[3] * qi[3]);
    double d = np_max(n, 1e-12);
    double x = qi[0] / d, y = qi[1] / d, z = qi[2] / d, w = qi[3] / d;
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

// ---------------------------------------------------------------------------
// box-box: 15-axis SAT, reference/incident face clip, 4-point reduction
// (_collide_native.pyx:20-263)
// ---------------------------------------------------------------------------
__device__ inline int face_axis(const double *R, const double *dir, double *sign) {
    double best = -1.0;
    int axis = 0;
    for (int m = 0; m < 3; m++) {
        double dv = R[m] * dir[0] + R[3 + m] * dir[1] + R[6 + m] * dir[2];
        if (fabs(dv) > best) {
            best = fabs(dv);
            axis = m;
            *sign = dv >= 0.0 ? 1.0 : -1.0;
        }
    }
    return axis;
}

__device__ inline void face_vertices(const double *c, const double *R, const double *h, int axis,
                                     double sign, double *verts) {
    int o0 = axis == 0 ? 1 : 0;
    int o1 = axis == 2 ? 1 : 2;
    double fc[3], u[3], v[3];
    for (int r = 0; r < 3; r++) {
        fc[r] = c[r] + R[r * 3 + axis] * sign * h[axis];
        u[r] = R[r * 3 + o0] * h[o0];
        v[r] = R[r * 3 + o1] * h[o1];
    }
    for (int r = 0; r < 3; r++) {
        verts[r] = fc[r] + u[r] + v[r];
        verts[3 + r] = fc[r] - u[r] + v[r];
        verts[6 + r] = fc[r] - u[r] - v[r];
        verts[9 + r] = fc[r] + u[r] - v[r];
    }
}

// keep up to 4 well-spread points (_collide_native.pyx:212-263)
__device__ inline int reduce4(const double *P, const double *dep, int nc, double *out_p,
                              double *out_d) {
    if (nc <= 4) {
        for (int i = 0; i < nc; i++) {
            out_p[i * 3] = P[i * 3]; out_p[i * 3 + 1] = P[i * 3 + 1]; out_p[i * 3 + 2] = P[i * 3 + 2];
            out_d[i] = dep[i];
        }
        return nc;
    }
    int k0 = 0;
    double best = P[0];
    for (int i = 1; i < nc; i++)
        if (P[i * 3] > best) { best = P[i * 3]; k0 = i; }
    int k1 = 0;
    best = -1.0;
    for (int i = 0; i < nc; i++) {
        double dd = 0.0;
        for (int r = 0; r < 3; r++) { double t = P[i * 3 + r] - P[k0 * 3 + r]; dd += t * t; }
        if (dd > best) { best = dd; k1 = i; }
    }
    int k2 = 0;
    best = -1.0;
    for (int i = 0; i < nc; i++) {
        double s1 = 0.0, s0 = 0.0;
        for (int r = 0; r < 3; r++) {
            double t = P[i * 3 + r] - P[k1 * 3 + r]; s1 += t * t;
            t = P[i * 3 + r] - P[k0 * 3 + r]; s0 += t * t;
        }
        double sc = sqrt(s1) + sqrt(s0);
        if (sc > best) { best = sc; k2 = i; }
    }
    int k3 = 0;
    best = -1.0;
    for (int i = 0; i < nc; i++) {
        double dd = 0.0;
        for (int r = 0; r < 3; r++) { double t = P[i * 3 + r] - P[k2 * 3 + r]; dd += t * t; }
        double sc = sqrt(dd);
        if (sc > best) { best = sc; k3 = i; }
    }
    int keep[4] = {k0, k1, k2, k3};
    int nk = 0;
    for (int i = 0; i < 4; i++) {
        bool dup = false;
        for (int j = 0; j < nk; j++) dup |= keep[i] == keep[j];
        if (!dup) keep[nk++] = keep[i];
    }
    for (int i = 0; i < nk; i++) {
        for (int r = 0; r < 3; r++) out_p[i * 3 + r] = P[keep[i] * 3 + r];
        out_d[i] = dep[keep[i]];
    }
    return nk;
}

__device__ inline int clip_faces(const double *ca, const double *Ra, const double *ha,
                                 const double *cb, const double *Rb, const double *hb,
                                 const double *nrm, double depth, double *out_p, double *out_d) {
    double a_align = -1.0, b_align = -1.0;
    for (int m = 0; m < 3; m++) {
        double dv = fabs(Ra[m] * nrm[0] + Ra[3 + m] * nrm[1] + Ra[6 + m] * nrm[2]);
        if (dv > a_align) a_align = dv;
        dv = fabs(Rb[m] * nrm[0] + Rb[3 + m] * nrm[1] + Rb[6 + m] * nrm[2]);
        if (dv > b_align) b_align = dv;
    }
    const bool flip = !(a_align >= b_align);
    const double *rc = flip ? cb : ca, *rR = flip ? Rb : Ra, *rh = flip ? hb : ha;
    const double *ic = flip ? ca : cb, *iR = flip ? Ra : Rb, *ih = flip ? ha : hb;
    double ref_n[3], neg[3];
    for (int r = 0; r < 3; r++) ref_n[r] = flip ? -nrm[r] : nrm[r];
    for (int r = 0; r < 3; r++) neg[r] = -ref_n[r];
    double isign = 0.0, rsign = 0.0;
    int iaxis = face_axis(iR, neg, &isign);
    // two polygon buffers used in turn (each clip reads one and writes the
    // other); the contact points then go into the one not holding the polygon
    double bufs[2][16 * 3];
    int cur_b = 0;
    int np_ = 4;
    face_vertices(ic, iR, ih, iaxis, isign, bufs[0]);
    int raxis = face_axis(rR, ref_n, &rsign);
    double refv[12];
    face_vertices(rc, rR, rh, raxis, rsign, refv);
    const double fp0 = refv[0], fp1 = refv[1], fp2 = refv[2];
    for (int other = 0; other < 3 && np_ > 0; other++) {
        if (other == raxis) continue;
        for (int si = 0; si < 2; si++) {
            double s = si == 0 ? 1.0 : -1.0;
            double pn0 = rR[other] * s, pn1 = rR[3 + other] * s, pn2 = rR[6 + other] * s;
            double offset = (rc[0] * pn0 + rc[1] * pn1 + rc[2] * pn2) + rh[other];
            const double *poly = bufs[cur_b];
            double *buf = bufs[cur_b ^ 1];
            int nb = 0;
            for (int i = 0; i < np_; i++) {
                const double *cur = &poly[i * 3];
                const double *nxt = &poly[((i + 1) % np_) * 3];
                double dc = pn0 * cur[0] + pn1 * cur[1] + pn2 * cur[2] - offset;
                double dn = pn0 * nxt[0] + pn1 * nxt[1] + pn2 * nxt[2] - offset;
                if (dc <= 0.0 && nb < 16) {
                    buf[nb * 3] = cur[0]; buf[nb * 3 + 1] = cur[1]; buf[nb * 3 + 2] = cur[2];
                    nb++;
                }
                if (dc * dn < 0.0 && nb < 16) {
                    double t = dc / (dc - dn);
                    for (int r = 0; r < 3; r++) buf[nb * 3 + r] = cur[r] + t * (nxt[r] - cur[r]);
                    nb++;
                }
            }
            np_ = nb;
            cur_b ^= 1;
            if (np_ == 0) break;
        }
    }
    const double *poly = bufs[cur_b];
    double *allp = bufs[cur_b ^ 1], alld[16];
    int nc = 0;
    for (int i = 0; i < np_; i++) {
        const double *p = &poly[i * 3];
        double pen = (fp0 - p[0]) * ref_n[0] + (fp1 - p[1]) * ref_n[1] + (fp2 - p[2]) * ref_n[2];
        if (pen >= -1e-6) {
            for (int r = 0; r < 3; r++) allp[nc * 3 + r] = p[r] + ref_n[r] * pen;
            alld[nc] = pen > 0.0 ? pen : 0.0;
            nc++;
        }
    }
    if (nc == 0) {
        for (int r = 0; r < 3; r++) out_p[r] = 0.5 * (ca[r] + cb[r]);
        out_d[0] = depth;
        return 1;
    }
    return reduce4(allp, alld, nc, out_p, out_d);
}

// the separating-axis part of box_box: false when separated, else the
// contact normal (A -> B) and the minimum overlap
// the best axis so far of the separating-axis test: the smallest overlap and
// its axis, signed to point from A to B
struct SatBest {
    double depth, x, y, z;
};
__device__ __forceinline__ void sat_begin(SatBest &b) { b.depth = 1e300; b.x = 0.0; b.y = 0.0; b.z = 0.0; }

// Axes k_lo .. k_hi - 1 of the 15 in the reference's order: A's columns, B's
// columns, then the normalised edge crosses A_i x B_j, skipped when
// |c|^2 <= EPS^2. False at the first separating axis; else b keeps the
// first axis of smallest overlap (strict <). Running 0..6 and then 6..15
// with the same b is the 15-axis loop.
__device__ inline bool sat_axes(int k_lo, int k_hi, const double *ca, const double *Ra, const double *ha,
                                const double *cb, const double *Rb, const double *hb, SatBest &b) {
    const double d0 = cb[0] - ca[0], d1 = cb[1] - ca[1], d2 = cb[2] - ca[2];
    for (int k = k_lo; k < k_hi; k++) {
        double a0, a1, a2;
        if (k < 3) { a0 = Ra[k]; a1 = Ra[3 + k]; a2 = Ra[6 + k]; }
        else if (k < 6) { a0 = Rb[k - 3]; a1 = Rb[k]; a2 = Rb[k + 3]; }
        else {
            int i = (k - 6) / 3, j = (k - 6) % 3;
            double cx = Ra[3 + i] * Rb[6 + j] - Ra[6 + i] * Rb[3 + j];
            double cy = Ra[6 + i] * Rb[j] - Ra[i] * Rb[6 + j];
            double cz = Ra[i] * Rb[3 + j] - Ra[3 + i] * Rb[j];
            double ln2 = cx * cx + cy * cy + cz * cz;
            if (!(ln2 > EPS_COLLIDE * EPS_COLLIDE)) continue;
            double inv = 1.0 / sqrt(ln2);
            a0 = cx * inv; a1 = cy * inv; a2 = cz * inv;
        }
        double ra = (fabs(a0 * Ra[0] + a1 * Ra[3] + a2 * Ra[6]) * ha[0] +
                     fabs(a0 * Ra[1] + a1 * Ra[4] + a2 * Ra[7]) * ha[1] +
                     fabs(a0 * Ra[2] + a1 * Ra[5] + a2 * Ra[8]) * ha[2]);
        double rb = (fabs(a0 * Rb[0] + a1 * Rb[3] + a2 * Rb[6]) * hb[0] +
                     fabs(a0 * Rb[1] + a1 * Rb[4] + a2 * Rb[7]) * hb[1] +
                     fabs(a0 * Rb[2] + a1 * Rb[5] + a2 * Rb[8]) * hb[2]);
        double proj = a0 * d0 + a1 * d1 + a2 * d2;
        double overlap = ra + rb - fabs(proj);
        if (overlap < 0.0) return false;
        if (overlap < b.depth) {
            b.depth = overlap;
            if (proj >= 0.0) { b.x = a0; b.y = a1; b.z = a2; }
            else { b.x = -a0; b.y = -a1; b.z = -a2; }
        }
    }
    return true;
}

__device__ inline bool box_box_sat(const double *ca, const double *Ra, const double *ha,
                                   const double *cb, const double *Rb, const double *hb,
                                   double *normal, double &depth) {
    SatBest b;
    sat_begin(b);
    normal[0] = normal[1] = normal[2] = 0.0;
    if (!sat_axes(0, 15, ca, Ra, ha, cb, Rb, hb, b)) return false;
    normal[0] = b.x; normal[1] = b.y; normal[2] = b.z;
    depth = b.depth;
    return true;
}

__device__ inline int box_box(const double *ca, const double *Ra, const double *ha,
                              const double *cb, const double *Rb, const double *hb,
                              double *normal, double *pts, double *deps) {
    double depth;
    if (!box_box_sat(ca, Ra, ha, cb, Rb, hb, normal, depth)) return 0;
    return clip_faces(ca, Ra, ha, cb, Rb, hb, normal, depth, pts, deps);
}

// _collide_native.pyx:285-299
__device__ inline int sphere_sphere(const double *ca, double ra, const double *cb, double rb,
                                    double *normal, double *pts, double *deps) {
    double dx = cb[0] - ca[0], dy = cb[1] - ca[1], dz = cb[2] - ca[2];
    double dist = sqrt(dx * dx + dy * dy + dz * dz);
    double r = ra + rb;
    if (dist >= r) return 0;
    double nx = 0.0, ny = 1.0, nz = 0.0;
    if (dist > EPS_COLLIDE) { nx = dx / dist; ny = dy / dist; nz = dz / dist; }
    double depth = r - dist;
    double f = ra - 0.5 * depth;
    normal[0] = nx; normal[1] = ny; normal[2] = nz;
    pts[0] = ca[0] + nx * f; pts[1] = ca[1] + ny * f; pts[2] = ca[2] + nz * f;
    deps[0] = depth;
    return 1;
}

// _collide_native.pyx:302-344; normal returned sphere -> box
__device__ inline int sphere_box(const double *cs, double rs, const double *cb, const double *Rb,
                                 const double *hb, double *normal, double *pts, double *deps) {
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
    deps[0] = depth;
    return 1;
}

}  // namespace omi
