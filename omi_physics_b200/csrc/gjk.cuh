// GJK intersection + EPA penetration for convex proxies (gjk.py:39-264,
// body.py:33-132), one warp per pair.
//
// All 32 lanes run the same scalar control flow on identical values; the
// lanes split the two loops that scale with the input: the support search
// over a convex hull's points (argmax with the lowest index winning ties, as
// np.argmax does) and the closest-face search over the polytope (first
// minimum in face order, as gjk._closest_face's strict '<' does). The
// polytope (vertices with their witnesses, faces, horizon edges) lives in
// shared memory and is written by lane 0 only, followed by __syncwarp().
#pragma once
#include "geometry.cuh"

namespace omi {

// Lanes cooperating on one pair. Host builds of this header (a test-only
// emulation that checks the device geometry against the oracle on the CPU)
// run the warp as a single lane.
// The support search, the simplex cases, the face distance, the serial
// rebuild and the contact point are called out of line on the device: inlined
// at every call site they made k_gjk large enough that its warps mostly waited
// on instruction fetch, and held 218 registers a thread (two blocks an SM);
// out of line it takes 165 (three blocks) and GJK/EPA runs 20-25% faster on
// the hull pile, with the same arithmetic.
#ifdef OMI_HOST_EMULATION
constexpr int WARP_LANES = 1;
#define GJK_OUTLINE inline
#else
constexpr int WARP_LANES = 32;
#define GJK_OUTLINE __noinline__
#endif

// Polytope bounds: 64 EPA iterations add at most 64 vertices; faces and
// horizon edges are bounded as the oracle bounds them. Rounded Minkowski sums
// (capsules, spheres against hulls) need more than 2V - 4 faces when nearly
// coplanar faces make the visible set ragged.
constexpr int EPA_V = 4 + 64 + 1;
constexpr int EPA_F = 512;
constexpr int EPA_E = 3 * EPA_F;

struct Proxy {
    int kind;              // 1 sphere, 2 box, 3 convex, 4 capsule, 5 triangle (local = 3 world vertices)
    double c[3], R[9], h[3], r;
    double e0[3], e1[3];   // capsule segment ends
    const double *local;   // convex local points (global memory)
    int m;
};

// Vertex indices are below EPA_V, so faces and edges are stored as bytes.
// The lanes' rebuild marks the directed edges of the visible faces in a
// bit table indexed by (from, to) and writes the new face list into F2.
constexpr int EPA_EDGE_WORDS = (EPA_V * EPA_V + 31) / 32;
struct EpaWork {
    double V[EPA_V][9];    // Minkowski point v, witness a, witness b
    unsigned char F[EPA_F][3];
    unsigned char E[EPA_E][2];
    unsigned char Ealive[EPA_E];
    unsigned char F2[EPA_F][3];
    unsigned int seen[EPA_EDGE_WORDS];   // zero between rebuilds
};
static_assert(EPA_V <= 256, "face and edge vertex indices are stored as bytes");

__device__ inline unsigned lane_id() { return threadIdx.x % WARP_LANES; }

// Warp-wide max / min of a double (NaN-free inputs) and min of an index.
// Ties are resolved by exact equality against the reduced value followed by
// an integer minimum, so the winner is the lowest index among equal values.
__device__ inline double warp_max(double x) {
    for (int off = 16; off > 0; off >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, off));
    return x;
}
__device__ inline double warp_min(double x) {
    for (int off = 16; off > 0; off >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, off));
    return x;
}
__device__ inline int warp_min_index(int i) {
#ifdef OMI_HOST_EMULATION
    return i;
#else
    return __reduce_min_sync(0xffffffffu, i);
#endif
}

// Proxy.support(d) (body.py:46-48, 69-73, 100-104, 125-128, 146-148)
__device__ GJK_OUTLINE void support(const Proxy &p, const double *d, double *out) {
    if (p.kind == 1) {
        double u[3];
        normalize3(d, u);
        for (int k = 0; k < 3; k++) out[k] = p.c[k] + p.r * u[k];
    } else if (p.kind == 2) {
        double s[3];
        for (int j = 0; j < 3; j++) {
            double col[3] = {p.R[j], p.R[3 + j], p.R[6 + j]};
            double l = dot_blas(col, d);
            double sg = l > 0 ? 1.0 : (l < 0 ? -1.0 : (l == 0 ? 0.0 : l));
            s[j] = sg * p.h[j];
        }
        for (int k = 0; k < 3; k++) out[k] = p.c[k] + gemv_row(&p.R[k * 3], s);
    } else if (p.kind == 5) {
        // TriangleProxy.support (body.py:146-148): the first vertex of the
        // largest verts @ d
        int best = 0;
        double bv = gemv_row(&p.local[0], d);
        for (int i = 1; i < 3; i++) {
            const double v = gemv_row(&p.local[i * 3], d);
            if (v > bv) { bv = v; best = i; }
        }
        for (int k = 0; k < 3; k++) out[k] = p.local[best * 3 + k];
    } else if (p.kind == 4) {
        // the segment end farther along d (the second on ties), plus radius
        const double *end = dot_blas(p.e0, d) > dot_blas(p.e1, d) ? p.e0 : p.e1;
        double u[3];
        normalize3(d, u);
        for (int k = 0; k < 3; k++) out[k] = end[k] + p.r * u[k];
    } else {
        // world = local @ R.T + center; argmax(world @ d), first index on ties:
        // warp max of the values, then the lowest index holding that value;
        // every lane then recomputes that world point with the same arithmetic
        const unsigned lane = lane_id();
        double best = -INFINITY;
        int bi = -1;
        for (int i = lane; i < p.m; i += WARP_LANES) {
            const double *l = &p.local[i * 3];
            double wpt[3];
            for (int k = 0; k < 3; k++) wpt[k] = dot_blas(l, &p.R[k * 3]) + p.c[k];
            const double v = gemv_row(wpt, d);
            if (bi < 0 || v > best) { best = v; bi = i; }
        }
        const double m = warp_max(best);
        const int win = warp_min_index((bi >= 0 && best == m) ? bi : 0x7fffffff);
        const int pick = win == 0x7fffffff ? 0 : win;
        const double *l = &p.local[pick * 3];
        for (int k = 0; k < 3; k++) out[k] = dot_blas(l, &p.R[k * 3]) + p.c[k];
    }
}

__device__ inline void center_hint(const Proxy &p, double *out) {
    if (p.kind == 5) {                     // verts.mean(axis=0) (body.py:150-152)
        for (int k = 0; k < 3; k++) out[k] = ((p.local[k] + p.local[3 + k]) + p.local[6 + k]) / 3.0;
        return;
    }
    if (p.kind != 3) { out[0] = p.c[0]; out[1] = p.c[1]; out[2] = p.c[2]; return; }
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;   // mean(axis=0): sequential row sum
    for (int i = 0; i < p.m; i++) {
        const double *l = &p.local[i * 3];
        s0 = s0 + (dot_blas(l, &p.R[0]) + p.c[0]);
        s1 = s1 + (dot_blas(l, &p.R[3]) + p.c[1]);
        s2 = s2 + (dot_blas(l, &p.R[6]) + p.c[2]);
    }
    out[0] = s0 / (double)p.m; out[1] = s1 / (double)p.m; out[2] = s2 / (double)p.m;
}

struct Vt { double v[3], a[3], b[3]; };

__device__ inline void mink(const Proxy &A, const Proxy &B, const double *d, Vt &o) {
    double nd[3] = {-d[0], -d[1], -d[2]};
    support(A, d, o.a);
    support(B, nd, o.b);
    sub3(o.a, o.b, o.v);
}

// ---- GJK simplex handling (gjk.py:60-117); s[] in the reference's list order
__device__ GJK_OUTLINE void do_line(Vt *s, int &n, double *d) {
    Vt b = s[0], a = s[1];
    double ab[3], ao[3];
    sub3(b.v, a.v, ab); neg3(a.v, ao);
    if (dot_blas(ab, ao) > 0) {
        double t[3];
        cross_np(ab, ao, t); cross_np(t, ab, d);
        if (dot_blas(d, d) < EPS_GJK) {
            double ax[3] = {0.0, 1.0, 0.0};
            if (fabs(ab[0]) < 0.9) { ax[0] = 1.0; ax[1] = 0.0; }
            cross_np(ab, ax, d);
        }
        s[0] = b; s[1] = a; n = 2;
        return;
    }
    s[0] = a; n = 1;
    d[0] = ao[0]; d[1] = ao[1]; d[2] = ao[2];
}

__device__ GJK_OUTLINE void do_triangle(Vt *s, int &n, double *d) {
    Vt c = s[0], b = s[1], a = s[2];
    double ab[3], ac[3], ao[3], abc[3], t[3];
    sub3(b.v, a.v, ab); sub3(c.v, a.v, ac); neg3(a.v, ao);
    cross_np(ab, ac, abc);
    cross_np(abc, ac, t);
    if (dot_blas(t, ao) > 0) {
        if (dot_blas(ac, ao) > 0) {
            double u[3];
            cross_np(ac, ao, u); cross_np(u, ac, d);
            s[0] = c; s[1] = a; n = 2;
            return;
        }
        s[0] = b; s[1] = a; n = 2;
        do_line(s, n, d);
        return;
    }
    cross_np(ab, abc, t);
    if (dot_blas(t, ao) > 0) {
        s[0] = b; s[1] = a; n = 2;
        do_line(s, n, d);
        return;
    }
    if (dot_blas(abc, ao) > 0) {
        s[0] = c; s[1] = b; s[2] = a; n = 3;
        d[0] = abc[0]; d[1] = abc[1]; d[2] = abc[2];
        return;
    }
    s[0] = b; s[1] = c; s[2] = a; n = 3;
    neg3(abc, d);
}

__device__ GJK_OUTLINE bool do_tetra(Vt *s, int &n, double *dir) {
    Vt d = s[0], c = s[1], b = s[2], a = s[3];
    double ab[3], ac[3], ad[3], ao[3], abc[3], acd[3], adb[3];
    sub3(b.v, a.v, ab); sub3(c.v, a.v, ac); sub3(d.v, a.v, ad); neg3(a.v, ao);
    cross_np(ab, ac, abc); cross_np(ac, ad, acd); cross_np(ad, ab, adb);
    if (dot_blas(abc, ao) > 0) { s[0] = c; s[1] = b; s[2] = a; n = 3; do_triangle(s, n, dir); return false; }
    if (dot_blas(acd, ao) > 0) { s[0] = d; s[1] = c; s[2] = a; n = 3; do_triangle(s, n, dir); return false; }
    if (dot_blas(adb, ao) > 0) { s[0] = b; s[1] = d; s[2] = a; n = 3; do_triangle(s, n, dir); return false; }
    dir[0] = dir[1] = dir[2] = 0.0;
    return true;
}

// gjk_intersect (gjk.py:39-57)
__device__ inline bool gjk(const Proxy &A, const Proxy &B, Vt *s, int &n) {
    double zero[3] = {0.0, 0.0, 0.0}, pa[3], pb[3], d[3], nd[3];
    support(B, zero, pb);
    support(A, zero, pa);
    sub3(pb, pa, d);
    if (dot_blas(d, d) < EPS_GJK) { d[0] = 1.0; d[1] = 0.0; d[2] = 0.0; }
    neg3(d, nd);
    mink(A, B, nd, s[0]);
    n = 1;
    neg3(s[0].v, d);
    for (int it = 0; it < 32; it++) {
        if (dot_blas(d, d) < EPS_GJK) return true;
        Vt wv;
        mink(A, B, d, wv);
        if (dot_blas(wv.v, d) < 0) return false;
        s[n++] = wv;
        if (n == 2) do_line(s, n, d);
        else if (n == 3) do_triangle(s, n, d);
        else if (do_tetra(s, n, d)) return true;
    }
    return false;
}

__device__ inline void put_vertex(EpaWork &W, int i, const Vt &x) {
    if (lane_id() == 0) {
        for (int k = 0; k < 3; k++) { W.V[i][k] = x.v[k]; W.V[i][3 + k] = x.a[k]; W.V[i][6 + k] = x.b[k]; }
    }
    __syncwarp();
}

// _closest_face (gjk.py:176-194): lanes split faces, first minimum wins
__device__ GJK_OUTLINE bool face_distance(const EpaWork &W, int f, double *nr, double *dd) {
    const double *a = W.V[W.F[f][0]], *b = W.V[W.F[f][1]], *c = W.V[W.F[f][2]];
    double e1[3], e2[3];
    sub3(b, a, e1); sub3(c, a, e2);
    cross_np(e1, e2, nr);
    const double ln = sqrt(dot_blas(nr, nr));
    if (ln < EPS_GJK) return false;
    for (int q = 0; q < 3; q++) nr[q] = nr[q] / ln;
    double d = dot_blas(nr, a);
    if (d < 0) { neg3(nr, nr); d = -d; }
    *dd = d;
    return d == d;            // a NaN distance never compares below the best
}

__device__ inline int closest_face(const EpaWork &W, int nf, double *bn, double *bd) {
    int best = -1;
    double best_d = INFINITY;
    for (int f = lane_id(); f < nf; f += WARP_LANES) {
        double nr[3], dd;
        if (face_distance(W, f, nr, &dd) && dd < best_d) { best = f; best_d = dd; }
    }
    const double m = warp_min(best_d);
    const int win = warp_min_index((best >= 0 && best_d == m) ? best : 0x7fffffff);
    if (win == 0x7fffffff) return -1;
    double nr[3], dd = 0.0;
    face_distance(W, win, nr, &dd);
    bn[0] = nr[0]; bn[1] = nr[1]; bn[2] = nr[2];
    *bd = dd;
    return win;
}

// _rebuild (gjk.py:197-217) by lane 0 alone: the ordered horizon-edge
// dictionary as the reference keeps it. Returns the new face count or -1
// when the bounded storage (at most `face_cap` <= EPA_F faces) would overflow.
__device__ GJK_OUTLINE int rebuild_serial(EpaWork &W, int nf, int ni, int face_cap = EPA_F) {
    int out = 0;
    if (lane_id() == 0) {
        const double *w = W.V[ni];
        int ne = 0, nk = 0;
        bool bad = false;
        for (int f = 0; f < nf && !bad; f++) {
            const double *a = W.V[W.F[f][0]];
            double e1[3], e2[3], nr[3], wa[3];
            sub3(W.V[W.F[f][1]], a, e1); sub3(W.V[W.F[f][2]], a, e2);
            cross_np(e1, e2, nr);
            sub3(w, a, wa);
            if (dot_blas(nr, wa) > 0) {
                int es[3][2] = {{W.F[f][0], W.F[f][1]}, {W.F[f][1], W.F[f][2]}, {W.F[f][2], W.F[f][0]}};
                for (int e = 0; e < 3; e++) {
                    int rev = -1, same = -1;
                    for (int q = 0; q < ne; q++) {
                        if (!W.Ealive[q]) continue;
                        if (W.E[q][0] == es[e][1] && W.E[q][1] == es[e][0]) rev = q;
                        if (W.E[q][0] == es[e][0] && W.E[q][1] == es[e][1]) same = q;
                    }
                    if (rev >= 0) W.Ealive[rev] = 0;
                    else if (same < 0) {
                        if (ne >= EPA_E) { bad = true; break; }
                        W.E[ne][0] = es[e][0]; W.E[ne][1] = es[e][1]; W.Ealive[ne] = 1; ne++;
                    }
                }
            } else {
                // kept faces compact in place: nk <= f, so face f is read before
                // any later write reaches its slot
                W.F[nk][0] = W.F[f][0]; W.F[nk][1] = W.F[f][1]; W.F[nk][2] = W.F[f][2]; nk++;
            }
        }
        for (int q = 0; q < ne && !bad; q++) {
            if (!W.Ealive[q]) continue;
            if (nk >= face_cap) { bad = true; break; }
            W.F[nk][0] = W.E[q][0]; W.F[nk][1] = W.E[q][1]; W.F[nk][2] = (unsigned char)ni; nk++;
        }
        out = bad ? -1 : nk;
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, out, 0);
}

#ifdef OMI_HOST_EMULATION
__device__ inline int rebuild(EpaWork &W, int nf, int ni, int face_cap = EPA_F) {
    return rebuild_serial(W, nf, ni, face_cap);
}
#else
__device__ __forceinline__ int edge_key(int u, int v) { return u * EPA_V + v; }

// _rebuild (gjk.py:197-217) with the lanes splitting the faces. The
// reference walks the faces that see the new point in order, and for each
// of a face's edges (a, b), (b, c), (c, a) deletes the reverse edge from an
// insertion-ordered dict if present, else inserts the edge; the surviving
// edges, in insertion order, each make a new face with the new point, after
// the faces that do not see it (in order). When no directed edge occurs
// twice among the visible faces (a closed polytope: every edge borders two
// faces), an edge survives exactly when its reverse is not among them, and
// its insertion order is its own place in the walk - both found in parallel
// from a bit table of the visible edges. A directed edge seen twice (a
// degenerate polytope) falls back to the dictionary walk of rebuild_serial.
__device__ inline int rebuild(EpaWork &W, int nf, int ni, int face_cap = EPA_F) {
    const unsigned lane = lane_id();
    const unsigned lt = (1u << lane) - 1u;
    const double *w = W.V[ni];
    bool dup = false;
    int nvis = 0;
    // visibility and the visible edges' bits
    for (int base = 0; base < nf; base += 32) {
        const int f = base + (int)lane;
        bool vis = false;
        if (f < nf) {
            const double *a = W.V[W.F[f][0]];
            double e1[3], e2[3], nr[3], wa[3];
            sub3(W.V[W.F[f][1]], a, e1); sub3(W.V[W.F[f][2]], a, e2);
            cross_np(e1, e2, nr);
            sub3(w, a, wa);
            vis = dot_blas(nr, wa) > 0;
        }
        if (vis) {
            for (int e = 0; e < 3; e++) {
                const int k = edge_key(W.F[f][e], W.F[f][(e + 1) % 3]);
                const unsigned bit = 1u << (k & 31);
                dup |= (atomicOr(&W.seen[k >> 5], bit) & bit) != 0;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, vis);
        if (lane == 0) reinterpret_cast<unsigned *>(W.E)[base >> 5] = m;   // visibility words (E as scratch)
        nvis += __popc(m);
    }
    __syncwarp();
    dup = __any_sync(0xffffffffu, dup);
    const unsigned *vmask = reinterpret_cast<const unsigned *>(W.E);
    int out = -1;
    if (!dup) {
        // kept faces, in order, then the surviving edges' new faces, in walk order
        const int K = nf - nvis;
        int nk = 0, ns = 0;
        for (int base = 0; base < nf; base += 32) {
            const int f = base + (int)lane;
            const unsigned m = vmask[base >> 5];
            const bool valid = f < nf, vis = valid && ((m >> lane) & 1u);
            const bool keep = valid && !vis;
            const unsigned km = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int pos = nk + __popc(km & lt);
                W.F2[pos][0] = W.F[f][0]; W.F2[pos][1] = W.F[f][1]; W.F2[pos][2] = W.F[f][2];
            }
            nk += __popc(km);
            int cnt = 0;
            bool surv[3] = {false, false, false};
            if (vis) {
                for (int e = 0; e < 3; e++) {
                    const int u = W.F[f][e], v = W.F[f][(e + 1) % 3];
                    const int k = edge_key(v, u);
                    surv[e] = !((W.seen[k >> 5] >> (k & 31)) & 1u);
                    cnt += surv[e];
                }
            }
            int pre = cnt;                                    // inclusive warp scan of the counts
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, pre, o);
                if ((int)lane >= o) pre += y;
            }
            int pos = K + ns + pre - cnt;
            for (int e = 0; e < 3; e++) {
                if (!surv[e]) continue;
                if (pos < face_cap) {
                    W.F2[pos][0] = W.F[f][e]; W.F2[pos][1] = W.F[f][(e + 1) % 3]; W.F2[pos][2] = (unsigned char)ni;
                }
                pos++;
            }
            ns += __shfl_sync(0xffffffffu, pre, 31);
        }
        out = K + ns > face_cap ? -1 : K + ns;
    }
    // clear the visible edges' bits for the next rebuild
    __syncwarp();
    for (int base = 0; base < nf; base += 32) {
        const int f = base + (int)lane;
        if (f < nf && ((vmask[base >> 5] >> lane) & 1u))
            for (int e = 0; e < 3; e++) {
                const int k = edge_key(W.F[f][e], W.F[f][(e + 1) % 3]);
                atomicAnd(&W.seen[k >> 5], ~(1u << (k & 31)));
            }
    }
    __syncwarp();
    if (dup) return rebuild_serial(W, nf, ni, face_cap);
    if (out > 0)
        for (int i = (int)lane; i < out; i += 32) { W.F[i][0] = W.F2[i][0]; W.F[i][1] = W.F2[i][1]; W.F[i][2] = W.F2[i][2]; }
    __syncwarp();
    return out;
}
#endif

// _contact_from_face + _barycentric (gjk.py:220-246)
__device__ GJK_OUTLINE void face_contact(const EpaWork &W, int f, const double *nrm, double dist,
                                   double *point) {
    const double *A = W.V[W.F[f][0]], *B = W.V[W.F[f][1]], *Cc = W.V[W.F[f][2]];
    double p[3] = {nrm[0] * dist, nrm[1] * dist, nrm[2] * dist};
    double v0[3], v1[3], v2[3];
    sub3(B, A, v0); sub3(Cc, A, v1); sub3(p, A, v2);
    double d00 = dot_blas(v0, v0), d01 = dot_blas(v0, v1), d11 = dot_blas(v1, v1);
    double d20 = dot_blas(v2, v0), d21 = dot_blas(v2, v1);
    double denom = d00 * d11 - d01 * d01;
    double bu = 1.0, bv = 0.0, bw = 0.0;
    if (!(fabs(denom) < EPS_GJK)) {
        bv = (d11 * d20 - d01 * d21) / denom;
        bw = (d00 * d21 - d01 * d20) / denom;
        bu = 1.0 - bv - bw;
    }
    for (int q = 0; q < 3; q++) {
        double pa = bu * A[3 + q] + bv * B[3 + q] + bw * Cc[3 + q];
        double pb = bu * A[6 + q] + bv * B[6 + q] + bw * Cc[6 + q];
        point[q] = 0.5 * (pa + pb);
    }
}

// epa (gjk.py:120-173). Returns 1 with normal/depth/point, 0 for None,
// -1 when bounded storage overflowed (reported, treated as None).
__device__ inline int epa(const Proxy &A, const Proxy &B, EpaWork &W, const Vt *s, int nv,
                          double *nrm, double *depth, double *point, int face_cap = EPA_F) {
    for (int i = 0; i < nv; i++) put_vertex(W, i, s[i]);
    if (nv < 4) {                                   // _expand_to_tetra
        Vt pts[4];
        for (int i = 0; i < nv; i++) pts[i] = s[i];
        int np_ = nv;
        const double dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        for (int k = 0; k < 6 && np_ < 4; k++) {
            Vt wv;
            mink(A, B, dirs[k], wv);
            bool ok = true;
            for (int p = 0; p < np_; p++) {
                double dv[3];
                sub3(wv.v, pts[p].v, dv);
                if (!(dot_blas(dv, dv) > EPS_GJK)) { ok = false; break; }
            }
            if (ok) pts[np_++] = wv;
        }
        if (np_ < 4) return 0;
        double e1[3], e2[3], e3[3], cr[3];
        sub3(pts[1].v, pts[0].v, e1); sub3(pts[2].v, pts[0].v, e2); sub3(pts[3].v, pts[0].v, e3);
        cross_np(e1, e2, cr);
        if (dot_blas(cr, e3) > 0) { Vt t = pts[1]; pts[1] = pts[2]; pts[2] = t; }
        for (int i = 0; i < 4; i++) put_vertex(W, i, pts[i]);
        nv = 4;
    }
    if (lane_id() == 0) {
        const int init[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 3, 2}};
        for (int f = 0; f < 4; f++) for (int k = 0; k < 3; k++) W.F[f][k] = init[f][k];
    }
    for (int i = lane_id(); i < EPA_EDGE_WORDS; i += WARP_LANES) W.seen[i] = 0u;
    __syncwarp();
    int nf = 4;
    double bn[3], bd;
    for (int it = 0; it < 64; it++) {
        int bf = closest_face(W, nf, bn, &bd);
        if (bf < 0) return 0;
        Vt wv;
        mink(A, B, bn, wv);
        double dd = dot_blas(wv.v, bn);
        if (dd - bd < 1e-6) {
            face_contact(W, bf, bn, bd, point);
            nrm[0] = bn[0]; nrm[1] = bn[1]; nrm[2] = bn[2]; *depth = bd;
            return 1;
        }
        if (nv >= EPA_V) return -1;
        put_vertex(W, nv, wv);
        nv++;
        nf = rebuild(W, nf, nv - 1, face_cap);
        if (nf < 0) return -1;
        if (nf == 0) return 0;
    }
    int bf = closest_face(W, nf, bn, &bd);
    if (bf < 0) return 0;
    face_contact(W, bf, bn, bd, point);
    nrm[0] = bn[0]; nrm[1] = bn[1]; nrm[2] = bn[2]; *depth = bd;
    return 1;
}

// collide_convex (gjk.py:249-264). Returns contacts (0/1), or -1 on overflow.
__device__ inline int collide_convex(const Proxy &A, const Proxy &B, EpaWork &W, double *normal,
                                     double *point, double *depth, int face_cap = EPA_F) {
    Vt s[4];
    int n = 0;
    if (!gjk(A, B, s, n)) return 0;
    double nr[3], dep, pt[3];
    int r = epa(A, B, W, s, n, nr, &dep, pt, face_cap);
    if (r <= 0) return r;
    double ha[3], hb[3], dc[3];
    center_hint(A, ha); center_hint(B, hb);
    sub3(hb, ha, dc);
    if (dot_blas(nr, dc) < 0) neg3(nr, nr);
    if (dep <= 1e-9) return 0;
    normalize3(nr, normal);
    point[0] = pt[0]; point[1] = pt[1]; point[2] = pt[2];
    *depth = dep;
    return 1;
}

}  // namespace omi
