// Capsule against batches of triangles: the compiled capsule_triangles of
// _collide_native.pyx:454-574 (the character controller's depenetration
// query, collide.py:438-462), for many capsules at once.
//
// Layout: q capsules as rows of 7 doubles (p0 xyz, p1 xyz, radius), the
// triangles of capsule c at [tri_off[c], tri_off[c+1]) of one (n, 3, 3)
// vertex array; outputs line up with the triangles (hit byte, point (3),
// normal (3), depth), zeros where there is no contact.
//
// One thread per triangle. Each warp takes tiles of 32 triangles: the tile's
// 72-byte vertex records are read with coalesced streaming loads into the
// warp's shared memory, each lane runs the face test on its triangle, the
// point / normal rows are written back through shared memory so every global
// store is coalesced, and the triangles the face test leaves open wait in a
// per-warp queue until 32 of them can take the rim test together.
// Per triangle 72 bytes are read and 57 written; the arithmetic (float64, in
// the reference's operation order, no contraction) is a few hundred
// operations, so the kernel sits near the HBM / FP64 ridge.
#pragma once
#include "geometry.cuh"

namespace omi {

constexpr int CT_THREADS = 128;   // threads of a block: four warps, each with its own tiles
constexpr int CT_CAP_DOUBLES = 7; // p0 (3), p1 (3), radius

// _dot3 (_collide_native.pyx:16-17): left to right
__device__ __forceinline__ double dot3_seq(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

// closest point on triangle abc to p: Ericson's Voronoi regions in the order
// _closest_on_tri tests them (_collide_native.pyx:364-410)
__device__ inline void tri_closest(const double *p, const double *a, const double *b, const double *c,
                                   double *out) {
    double ab[3], ac[3], ap[3];
#pragma unroll
    for (int m = 0; m < 3; m++) { ab[m] = b[m] - a[m]; ac[m] = c[m] - a[m]; ap[m] = p[m] - a[m]; }
    const double d1 = dot3_seq(ab, ap), d2 = dot3_seq(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { out[0] = a[0]; out[1] = a[1]; out[2] = a[2]; return; }
    double bp[3];
#pragma unroll
    for (int m = 0; m < 3; m++) bp[m] = p[m] - b[m];
    const double d3 = dot3_seq(ab, bp), d4 = dot3_seq(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { out[0] = b[0]; out[1] = b[1]; out[2] = b[2]; return; }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double v = d1 / (d1 - d3);
#pragma unroll
        for (int m = 0; m < 3; m++) out[m] = a[m] + v * ab[m];
        return;
    }
    double cp[3];
#pragma unroll
    for (int m = 0; m < 3; m++) cp[m] = p[m] - c[m];
    const double d5 = dot3_seq(ab, cp), d6 = dot3_seq(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; return; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double w = d2 / (d2 - d6);
#pragma unroll
        for (int m = 0; m < 3; m++) out[m] = a[m] + w * ac[m];
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
#pragma unroll
        for (int m = 0; m < 3; m++) out[m] = b[m] + w * (c[m] - b[m]);
        return;
    }
    const double inv = 1.0 / (va + vb + vc);
    const double v = vb * inv, w = vc * inv;
#pragma unroll
    for (int m = 0; m < 3; m++) out[m] = a[m] + ab[m] * v + ac[m] * w;
}

// closest points of segments p1q1 and p2q2 (_collide_native.pyx:413-451)
__device__ inline void seg_closest(const double *p1, const double *q1, const double *p2, const double *q2,
                                   double *o1, double *o2) {
    double d1[3], d2[3], r[3], s, t;
#pragma unroll
    for (int m = 0; m < 3; m++) { d1[m] = q1[m] - p1[m]; d2[m] = q2[m] - p2[m]; r[m] = p1[m] - p2[m]; }
    const double aa = dot3_seq(d1, d1), e = dot3_seq(d2, d2), f = dot3_seq(d2, r);
    if (aa <= EPS_COLLIDE && e <= EPS_COLLIDE) {
#pragma unroll
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
#pragma unroll
    for (int m = 0; m < 3; m++) { o1[m] = p1[m] + d1[m] * s; o2[m] = p2[m] + d2[m] * t; }
}

// One triangle against the capsule (collide.py:309-382 as compiled): over
// the face, the deepest cap end whose perpendicular foot lies on the triangle
// is pushed back to the side the capsule's centre is on, depth unbounded;
// otherwise the nearest of the cap ends to the triangle and of the axis to
// the three edges (first strict minimum), if nearer than the radius. In two
// phases: capsule_face decides the face case and leaves what the rim test
// reuses (the closest points on the triangle to the two cap ends - the face
// and rim tests ask for the same two - when it found them); capsule_rim
// answers the rest. Each returns 1 on contact, with the point on the
// triangle and the normal pointing from the triangle toward the capsule.
struct CapRim {
    double tpk[2][3];
    bool have_tp;
};

__device__ __forceinline__ void tri_face(const double *v0, const double *v1, const double *v2, double *face,
                                         double &face_len) {
    double e1[3], e2[3];
#pragma unroll
    for (int m = 0; m < 3; m++) { e1[m] = v1[m] - v0[m]; e2[m] = v2[m] - v0[m]; }
    face[0] = e1[1] * e2[2] - e1[2] * e2[1];
    face[1] = e1[2] * e2[0] - e1[0] * e2[2];
    face[2] = e1[0] * e2[1] - e1[1] * e2[0];
    face_len = sqrt(dot3_seq(face, face));
}

__device__ inline int capsule_face(const double *c0, const double *c1, const double *centre, double radius,
                                   const double *v0, const double *v1, const double *v2, CapRim &rim,
                                   double *point, double *normal, double *depth) {
    double face[3], face_len;
    tri_face(v0, v1, v2, face, face_len);
    rim.have_tp = false;
    if (!(face_len > EPS_COLLIDE)) return 0;
    double fn[3];
#pragma unroll
    for (int m = 0; m < 3; m++) fn[m] = face[m] / face_len;
    double g[3] = {centre[0] - v0[0], centre[1] - v0[1], centre[2] - v0[2]};
    if (fn[0] * g[0] + fn[1] * g[1] + fn[2] * g[2] < 0.0) {
        fn[0] = -fn[0]; fn[1] = -fn[1]; fn[2] = -fn[2];
    }
    bool found = false;
    double best = -1e300, bp[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const double *sp = k ? c1 : c0;
#pragma unroll
        for (int m = 0; m < 3; m++) g[m] = sp[m] - v0[m];
        const double h = fn[0] * g[0] + fn[1] * g[1] + fn[2] * g[2];
        double foot[3];
#pragma unroll
        for (int m = 0; m < 3; m++) foot[m] = sp[m] - fn[m] * h;
        double *tp = rim.tpk[k];
        tri_closest(sp, v0, v1, v2, tp);
#pragma unroll
        for (int m = 0; m < 3; m++) g[m] = foot[m] - tp[m];
        if (g[0] * g[0] + g[1] * g[1] + g[2] * g[2] > EPS_COLLIDE * EPS_COLLIDE) continue;
        const double reach = radius - h;
        if (reach > 0.0 && reach > best) {
            best = reach;
            found = true;
            bp[0] = tp[0]; bp[1] = tp[1]; bp[2] = tp[2];
        }
    }
    rim.have_tp = true;
    if (!found) return 0;
    *depth = best;
#pragma unroll
    for (int m = 0; m < 3; m++) { point[m] = bp[m]; normal[m] = fn[m]; }
    return 1;
}

__device__ inline int capsule_rim(const double *c0, const double *c1, double radius, const double *v0,
                                  const double *v1, const double *v2, CapRim &rim, double *point,
                                  double *normal, double *depth) {
    if (!rim.have_tp) {
        tri_closest(c0, v0, v1, v2, rim.tpk[0]);
        tri_closest(c1, v0, v1, v2, rim.tpk[1]);
    }
    double best_d2 = 1e300, bsp[3] = {0.0, 0.0, 0.0}, btp[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const double *sp = k ? c1 : c0;
        const double *tp = rim.tpk[k];
        const double gx = sp[0] - tp[0], gy = sp[1] - tp[1], gz = sp[2] - tp[2];
        const double d2 = gx * gx + gy * gy + gz * gz;
        if (d2 < best_d2) {
            best_d2 = d2;
#pragma unroll
            for (int m = 0; m < 3; m++) { bsp[m] = sp[m]; btp[m] = tp[m]; }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double *ea = k == 0 ? v0 : (k == 1 ? v1 : v2);
        const double *eb = k == 0 ? v1 : (k == 1 ? v2 : v0);
        double ax[3], ed[3];
        seg_closest(c0, c1, ea, eb, ax, ed);
        const double gx = ax[0] - ed[0], gy = ax[1] - ed[1], gz = ax[2] - ed[2];
        const double d2 = gx * gx + gy * gy + gz * gz;
        if (d2 < best_d2) {
            best_d2 = d2;
#pragma unroll
            for (int m = 0; m < 3; m++) { bsp[m] = ax[m]; btp[m] = ed[m]; }
        }
    }
    if (best_d2 >= radius * radius) return 0;
    const double dist = sqrt(best_d2);
    if (dist > EPS_COLLIDE) {
#pragma unroll
        for (int m = 0; m < 3; m++) normal[m] = (bsp[m] - btp[m]) / dist;
    } else {
        double face[3], face_len;
        tri_face(v0, v1, v2, face, face_len);
        if (face_len > EPS_COLLIDE) {
#pragma unroll
            for (int m = 0; m < 3; m++) normal[m] = face[m] / face_len;
        } else {
            normal[0] = normal[1] = normal[2] = 0.0;
        }
    }
    *depth = radius - dist;
#pragma unroll
    for (int m = 0; m < 3; m++) point[m] = btp[m];
    return 1;
}

__device__ inline int capsule_triangle(const double *c0, const double *c1, const double *centre, double radius,
                                       const double *v0, const double *v1, const double *v2, double *point,
                                       double *normal, double *depth) {
    CapRim rim;
    if (capsule_face(c0, c1, centre, radius, v0, v1, v2, rim, point, normal, depth)) return 1;
    return capsule_rim(c0, c1, radius, v0, v1, v2, rim, point, normal, depth);
}

// Host builds of this header (a test-only emulation that checks the per-
// triangle arithmetic against the oracle on the CPU) stop here.
#ifndef OMI_HOST_EMULATION

// the capsule owning triangle i: the largest c in [lo, hi] with off[c] <= i
// (reads off[lo + 1 .. hi] only)
__device__ __forceinline__ int capsule_of(const int64_t *off, int lo, int hi, int64_t i) {
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&off[mid]) <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// the same by a whole warp, 32 candidates a round (~4 rounds for 65536
// capsules instead of 16 dependent loads); every lane returns the answer.
// The range shrinks every round and every read stays in [lo, hi], whatever
// off holds.
__device__ __forceinline__ int capsule_of_warp(const int64_t *off, int lo, int hi, int64_t i, int lane) {
    while (hi > lo) {
        const int step = (hi - lo + 31) / 32;
        const int c = min(hi, lo + (lane + 1) * step);
        const int k = __popc(__ballot_sync(0xffffffffu, __ldg(&off[c]) <= i));
        const int nlo = k == 0 ? lo : min(hi, lo + k * step);
        const int nhi = k == 32 ? hi : min(hi, lo + (k + 1) * step - 1);
        lo = nlo;
        hi = max(nlo, nhi);
    }
    return lo;
}

constexpr int CT_WARPS = CT_THREADS / 32;
constexpr int CT_QUEUE = 64;          // rim items a warp holds (31 left over + 32 new at most)
constexpr int CT_QITEM = 15;          // vertices (9) and the two closest points (6)

// Triangles [0, n) of this launch are global triangles [base, base + n): the
// vertex and output pointers are the launch's own, the capsule ranges
// tri_off are global (a host pipeline launches one chunk at a time).
//
// Each warp takes tiles of 32 triangles (grid-stride): coalesced streaming
// loads of the tile's vertex records into the warp's shared memory, one
// triangle per lane through the face test, the tile's outputs written back
// through shared memory so every global store is coalesced. A triangle the
// face test does not decide goes to the warp's rim queue with what the rim
// test reuses; whenever the queue holds 32 items the whole warp runs the rim
// test on them, one per lane, and writes each answer over its triangle's
// slot. The two tests thus run on full warps instead of diverging lane by
// lane. Only __syncwarp orders a warp's work; there is no block barrier.
__global__ void __launch_bounds__(CT_THREADS) k_capsule_triangles(
    const double *__restrict__ caps, const int64_t *__restrict__ tri_off, int q,
    const double *__restrict__ verts, int64_t base, int64_t n, uint8_t *__restrict__ hit,
    double *__restrict__ points, double *__restrict__ normals, double *__restrict__ depths) {
    __shared__ double sv[CT_WARPS][32 * 9];      // the tile's vertices, then its point / normal rows
    __shared__ double qd[CT_WARPS][CT_QUEUE * CT_QITEM];
    __shared__ int64_t qt[CT_WARPS][CT_QUEUE];
    __shared__ int qc[CT_WARPS][CT_QUEUE];
    __shared__ unsigned char qh[CT_WARPS][CT_QUEUE];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *wv = sv[wib], *wq = qd[wib];
    int64_t *wt = qt[wib];
    int *wc = qc[wib];
    unsigned char *wh = qh[wib];
    int queued = 0;
    // the rim test on queue items [from, from + count), one per lane
    auto drain = [&](int from, int count) {
        if (lane < count) {
            const int e = from + lane;
            const double *it = &wq[e * CT_QITEM];
            const double *cp = caps + (size_t)wc[e] * CT_CAP_DOUBLES;
            double c0[3], c1[3];
#pragma unroll
            for (int k = 0; k < 3; k++) { c0[k] = __ldg(&cp[k]); c1[k] = __ldg(&cp[3 + k]); }
            double v[9];
#pragma unroll
            for (int k = 0; k < 9; k++) v[k] = it[k];
            CapRim rim;
            rim.have_tp = wh[e] != 0;
#pragma unroll
            for (int k = 0; k < 3; k++) { rim.tpk[0][k] = it[9 + k]; rim.tpk[1][k] = it[12 + k]; }
            double pt[3], nr[3], dep;
            const int h = capsule_rim(c0, c1, __ldg(&cp[6]), v, v + 3, v + 6, rim, pt, nr, &dep);
            if (h) {
                const int64_t t = wt[e];
                hit[t] = 1;
#pragma unroll
                for (int k = 0; k < 3; k++) { points[t * 3 + k] = pt[k]; normals[t * 3 + k] = nr[k]; }
                depths[t] = dep;
            }
        }
        __syncwarp();
    };
    const int64_t stride = (int64_t)gridDim.x * CT_THREADS;
    for (int64_t t0 = ((int64_t)blockIdx.x * CT_WARPS + wib) * 32; t0 < n; t0 += stride) {
        const int m = (int)(n - t0 < 32 ? n - t0 : 32);
        const double *src = verts + t0 * 9;
        for (int j = lane; j < m * 9; j += 32) wv[j] = __ldcs(src + j);
        const int first = capsule_of_warp(tri_off, 0, q - 1, base + t0, lane);
        const int last = capsule_of_warp(tri_off, first, q - 1, base + t0 + m - 1, lane);
        __syncwarp();
        bool defer = false;
        int c = 0;
        CapRim rim;
        double pt[3] = {0.0, 0.0, 0.0}, nr[3] = {0.0, 0.0, 0.0}, dep = 0.0;
        if (lane < m) {
            c = capsule_of(tri_off, first, last, base + t0 + lane);
            const double *cp = caps + (size_t)c * CT_CAP_DOUBLES;
            double c0[3], c1[3], centre[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                c0[k] = __ldg(&cp[k]);
                c1[k] = __ldg(&cp[3 + k]);
                centre[k] = (c0[k] + c1[k]) * 0.5;
            }
            const double *v = &wv[lane * 9];
            const int h = capsule_face(c0, c1, centre, __ldg(&cp[6]), v, v + 3, v + 6, rim, pt, nr, &dep);
            defer = !h;
            hit[t0 + lane] = (uint8_t)h;
            __stcs(&depths[t0 + lane], dep);
        }
        // queue the undecided triangles, in lane order
        const unsigned dm = __ballot_sync(0xffffffffu, defer);
        if (defer) {
            const int e = queued + __popc(dm & ((1u << lane) - 1u));
            double *it = &wq[e * CT_QITEM];
#pragma unroll
            for (int k = 0; k < 9; k++) it[k] = wv[lane * 9 + k];
#pragma unroll
            for (int k = 0; k < 3; k++) { it[9 + k] = rim.tpk[0][k]; it[12 + k] = rim.tpk[1][k]; }
            wt[e] = t0 + lane;
            wc[e] = c;
            wh[e] = rim.have_tp ? 1 : 0;
        }
        queued += __popc(dm);
        __syncwarp();                                   // the queue has copied the vertices
        if (lane < m) {
#pragma unroll
            for (int k = 0; k < 3; k++) { wv[lane * 3 + k] = pt[k]; wv[96 + lane * 3 + k] = nr[k]; }
        }
        __syncwarp();
        for (int j = lane; j < m * 3; j += 32) {
            __stcs(&points[t0 * 3 + j], wv[j]);
            __stcs(&normals[t0 * 3 + j], wv[96 + j]);
        }
        __syncwarp();
        if (queued >= 32) {
            drain(queued - 32, 32);
            queued -= 32;
        }
    }
    if (queued > 0) drain(0, queued);
}

#endif  // OMI_HOST_EMULATION

}  // namespace omi
