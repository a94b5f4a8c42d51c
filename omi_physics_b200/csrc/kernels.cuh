// Kernels of one PhysicsWorld.step over every active world of an arena.
//
// Launch order inside a step (omi_b200.cu) differs from the reference's
// stage order in one place: integrate_forces runs after the broadphase
// instead of before refit. Refit, sort and the pair sweep read only poses,
// AABBs, motion types and awake flags, none of which integrate_forces
// changes, so the results are identical; the benefit is that a pair-buffer
// overflow is known before any body state is modified and the step can be
// re-run after the buffers grow.
#pragma once
#include "arena.cuh"
#include "geometry.cuh"
#include "gjk.cuh"

namespace omi {

constexpr int WF_SLEEP = 1, WF_WARM = 2, WF_COLLISION = 4;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ bool pairs_over(const Arena &A) {
    return A.pair_scan[A.NB] > A.pair_cap;
}
// pair or contact overflow; valid once the contact scan of this step ran
__device__ __forceinline__ bool overflowed(const Arena &A) {
    if (A.pair_scan[A.NB] > A.pair_cap) return true;
    return A.contact_scan[A.pair_scan[A.NB]] > A.contact_cap;
}
__device__ __forceinline__ bool world_collides(const Arena &A, int w) {
    return A.w_active[w] && (A.w_flags[w] & WF_COLLISION);
}
__device__ __forceinline__ bool dyn(const Arena &A, int i) { return A.mtype[i] == 2; }

// ---------------------------------------------------------------------------
// refit: world AABBs (world.py:471-508) and world inverse inertia
// einsum('nij,nkj->nik', R*invI, R) (solver.py:215-220), one thread per body
// ---------------------------------------------------------------------------
__global__ void k_refit(Arena A) {
    if (blockIdx.x == 0 && threadIdx.x == 0) A.gjk_n[0] = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.NB; i += gridDim.x * blockDim.x) {
        int w = A.body_world[i];
        if (!world_collides(A, w) || i - A.w_body_off[w] >= A.w_body_n[w]) continue;
        double R[9];
        quat_to_matrix(&A.q[i * 4], R);
        const double *h = &A.half[i * 3], *p = &A.pos[i * 3];
        const int kind = A.kind[i];
        double lo[3], hi[3];
        for (int r = 0; r < 3; r++) {
            double hw = (fabs(R[r * 3]) * h[0] + fabs(R[r * 3 + 2]) * h[2]) + fabs(R[r * 3 + 1]) * h[1];
            if (kind == 1) hw = h[r];
            lo[r] = (p[r] - hw) - 0.05;
            hi[r] = (p[r] + hw) + 0.05;
        }
        if (kind == 0) {
            for (int r = 0; r < 3; r++) lo[r] = hi[r] = p[r];
        } else if (kind == 3) {
            const int s = A.shape[i];
            const double *pts = &A.points[A.pt_off[s] * 3];
            const int m = A.pt_cnt[s];
            double mn[3], mx[3];
            for (int j = 0; j < m; j++) {
                for (int c = 0; c < 3; c++) {
                    double x = dot_blas(&pts[j * 3], &R[c * 3]) + p[c];
                    if (j == 0 || x < mn[c]) mn[c] = x;
                    if (j == 0 || x > mx[c]) mx[c] = x;
                }
            }
            for (int c = 0; c < 3; c++) { lo[c] = mn[c] - 0.05; hi[c] = mx[c] + 0.05; }
        }
        for (int r = 0; r < 3; r++) { A.aabb_min[i * 3 + r] = lo[r]; A.aabb_max[i * 3 + r] = hi[r]; }
        const double *ii = &A.inv_inertia[i * 3];
        double s[9];
        for (int r = 0; r < 3; r++)
            for (int j = 0; j < 3; j++) s[r * 3 + j] = R[r * 3 + j] * ii[j];
        double *W = &A.invIw[i * 9];
        for (int r = 0; r < 3; r++)
            for (int k = 0; k < 3; k++)
                W[r * 3 + k] = (s[r * 3] * R[k * 3] + s[r * 3 + 2] * R[k * 3 + 2]) + s[r * 3 + 1] * R[k * 3 + 1];
    }
}

// ---------------------------------------------------------------------------
// broadphase sort: np.argsort(min_x, kind='stable') per world
// (broadphase.py:261). One CTA per world; merge sort on (key, index) pairs,
// the index breaking ties, so the result is the stable order. Each pass
// places every element by one binary search (its rank in the other run).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool key_less(double ka, int va, double kb, int vb) {
    return ka < kb || (!(kb < ka) && va < vb);
}

__global__ void k_sort(Arena A, int smem_cap) {
    extern __shared__ __align__(16) unsigned char smem[];
    for (int w = blockIdx.x; w < A.W; w += gridDim.x) {
        if (!world_collides(A, w)) continue;
        const int off = A.w_body_off[w], n = A.w_body_n[w];
        double *k0, *k1;
        int *v0, *v1;
        if (n <= smem_cap) {
            k0 = reinterpret_cast<double *>(smem);
            k1 = k0 + smem_cap;
            v0 = reinterpret_cast<int *>(k1 + smem_cap);
            v1 = v0 + smem_cap;
        } else {
            k0 = A.sort_k[0] + off; k1 = A.sort_k[1] + off;
            v0 = A.sort_v[0] + off; v1 = A.sort_v[1] + off;
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double x = A.aabb_min[(off + i) * 3];
            k0[i] = (x != x) ? INFINITY : x + 0.0;   // NaN sorts last; -0.0 == 0.0
            v0[i] = i;
        }
        __syncthreads();
        for (int width = 1; width < n; width <<= 1) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const int seg = (i / (2 * width)) * (2 * width);
                const int mid = min(seg + width, n), end = min(seg + 2 * width, n);
                const double key = k0[i];
                const int val = v0[i];
                int lo, hi, base;
                if (i < mid) { lo = mid; hi = end; base = i - seg; }
                else { lo = seg; hi = mid; base = i - mid; }
                const int start = lo;
                while (lo < hi) {
                    int m = (lo + hi) >> 1;
                    if (key_less(k0[m], v0[m], key, val)) lo = m + 1; else hi = m;
                }
                const int pos = seg + base + (lo - start);
                k1[pos] = key;
                v1[pos] = val;
            }
            __syncthreads();
            double *tk = k0; k0 = k1; k1 = tk;
            int *tv = v0; v0 = v1; v1 = tv;
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            A.order[off + i] = off + v0[i];
            A.sorted_x[off + i] = k0[i];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// sweep-and-prune windows (broadphase.py:262-294): for sorted row k the
// candidates are rows k+1 .. searchsorted(lo_sx, hi_sx[k], 'right')-1; keep
// y/z overlap (>=), at least one dynamic body and interacting filters. One
// warp per sorted row; lanes test 32 candidates at a time and a ballot keeps
// the reference's k-major, then kj, order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool pair_keep(const Arena &A, int w, int a, int b) {
    const double *la = &A.aabb_min[a * 3], *ha = &A.aabb_max[a * 3];
    const double *lb = &A.aabb_min[b * 3], *hb = &A.aabb_max[b * 3];
    bool keep = (ha[1] >= lb[1]) & (hb[1] >= la[1]) & (ha[2] >= lb[2]) & (hb[2] >= la[2]);
    keep &= (A.mtype[a] == 2) | (A.mtype[b] == 2);
    if (keep) {
        const int rows = A.w_filter_rows[w];
        keep = A.filter_matrix[A.w_filter_off[w] + A.filter_row[a] * rows + A.filter_row[b]] != 0;
    }
    return keep;
}

__device__ __forceinline__ int window_end(const Arena &A, int off, int end_w, double hx) {
    int lo = off, hi = end_w;
    while (lo < hi) {
        int m = (lo + hi) >> 1;
        if (A.sorted_x[m] <= hx) lo = m + 1; else hi = m;
    }
    return lo;
}

__global__ void k_pair_count(Arena A) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.NB; e += nwarps) {
        const int w = A.body_world[e];
        int cnt = 0;
        if (world_collides(A, w) && e - A.w_body_off[w] < A.w_body_n[w]) {
            const int off = A.w_body_off[w], end_w = off + A.w_body_n[w];
            const int a = A.order[e];
            const int endk = window_end(A, off, end_w, A.aabb_max[a * 3]);
            for (int base = e + 1; base < endk; base += 32) {
                const int kj = base + lane;
                bool keep = kj < endk && pair_keep(A, w, a, A.order[kj]);
                cnt += __popc(__ballot_sync(FULL, keep));
            }
        }
        if (lane == 0) A.pair_cnt[e] = cnt;
    }
}

__global__ void k_pair_emit(Arena A) {
    if (pairs_over(A)) return;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.NB; e += nwarps) {
        const int w = A.body_world[e];
        if (!world_collides(A, w) || e - A.w_body_off[w] >= A.w_body_n[w]) continue;
        const int off = A.w_body_off[w], end_w = off + A.w_body_n[w];
        const int a = A.order[e];
        const int endk = window_end(A, off, end_w, A.aabb_max[a * 3]);
        int out = A.pair_scan[e];
        for (int base = e + 1; base < endk; base += 32) {
            const int kj = base + lane;
            int b = -1;
            bool keep = false;
            if (kj < endk) { b = A.order[kj]; keep = pair_keep(A, w, a, b); }
            const unsigned m = __ballot_sync(FULL, keep);
            if (keep) {
                const int slot = out + __popc(m & ((1u << lane) - 1u));
                const int p = a < b ? a : b, q = a < b ? b : a;
                A.pair_a[slot] = p;
                A.pair_b[slot] = q;
                // solid-pair filter (world.py:663-670): both colliders and an awake mover
                const bool mp = (A.mtype[p] == 2 && A.awake[p]) || A.mtype[p] == 1;
                const bool mq = (A.mtype[q] == 2 && A.awake[q]) || A.mtype[q] == 1;
                A.pair_solid[slot] = (A.shape[p] >= 0 && A.shape[q] >= 0 && (mp || mq)) ? 1 : 0;
            }
            out += __popc(m);
        }
    }
}

// ---------------------------------------------------------------------------
// exclusive scan of n ints (n = *n_ptr when given), out[n] = total.
// Tiles of 4096 (1024 threads x 4) -> tile sums -> one-CTA scan -> add.
// ---------------------------------------------------------------------------
constexpr int SCAN_TILE = 4096;

__device__ inline int block_exclusive_scan(int v, int *sh, int *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    int res = x - v + (wid > 0 ? sh[wid - 1] : 0);
    if (total) *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return res;
}

__global__ void k_scan_tiles(const int *in, int *out, int n_const, const int *n_ptr,
                             const int *gate_scan, int gate_idx, int gate_cap, int *tile_sums) {
    __shared__ int sh[32];
    if (gate_scan && gate_scan[gate_idx] > gate_cap) return;
    const int n = n_ptr ? *n_ptr : n_const;
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * 4;
    int v[4], s = 0;
    for (int j = 0; j < 4; j++) { v[j] = (base + j < n) ? in[base + j] : 0; s += v[j]; }
    int total;
    int pre = block_exclusive_scan(s, sh, &total);
    for (int j = 0; j < 4; j++) {
        if (base + j < n) out[base + j] = pre;
        pre += v[j];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_top(int *tile_sums, int ntiles, const int *gate_scan, int gate_idx,
                           int gate_cap) {
    __shared__ int sh[32];
    if (gate_scan && gate_scan[gate_idx] > gate_cap) return;
    int carry = 0;
    for (int base = 0; base < ntiles; base += blockDim.x * 4) {
        const int i0 = base + threadIdx.x * 4;
        int v[4], s = 0;
        for (int j = 0; j < 4; j++) { v[j] = (i0 + j < ntiles) ? tile_sums[i0 + j] : 0; s += v[j]; }
        int total;
        int pre = block_exclusive_scan(s, sh, &total) + carry;
        for (int j = 0; j < 4; j++) {
            if (i0 + j < ntiles) tile_sums[i0 + j] = pre;
            pre += v[j];
        }
        carry += total;
    }
    if (threadIdx.x == 0) tile_sums[ntiles] = carry;
}

__global__ void k_scan_add(int *out, int n_const, const int *n_ptr, const int *tile_sums,
                           int ntiles, const int *gate_scan, int gate_idx, int gate_cap) {
    if (gate_scan && gate_scan[gate_idx] > gate_cap) return;
    const int n = n_ptr ? *n_ptr : n_const;
    const int base = blockIdx.x * SCAN_TILE;
    const int add = tile_sums[blockIdx.x];
    for (int j = threadIdx.x; j < SCAN_TILE; j += blockDim.x) {
        const int i = base + j;
        if (i < n) out[i] += add;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_sums[ntiles];
}

// record an overflow (the host regrows and re-runs the step)
__global__ void k_pair_check(Arena A) {
    if (A.pair_scan[A.NB] > A.pair_cap) {
        A.status[ST_OVERFLOW] = 1;
        A.status[ST_PAIRS_NEEDED] = A.pair_scan[A.NB];
    }
}
__global__ void k_contact_check(Arena A) {
    if (pairs_over(A)) return;
    const int K = A.contact_scan[A.pair_scan[A.NB]];
    if (K > A.contact_cap) {
        A.status[ST_OVERFLOW] = 2;
        A.status[ST_CONTACTS_NEEDED] = K;
    }
}

// ---------------------------------------------------------------------------
// integrate forces (backend.py:26-40) + prev pose copy (world.py:414-415)
// ---------------------------------------------------------------------------
__global__ void k_integrate_forces(Arena A, int gated) {
    if (gated && overflowed(A)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.NB; i += gridDim.x * blockDim.x) {
        const int w = A.body_world[i];
        if (!A.w_active[w] || i - A.w_body_off[w] >= A.w_body_n[w]) continue;
        for (int c = 0; c < 3; c++) A.prev_pos[i * 3 + c] = A.pos[i * 3 + c];
        for (int c = 0; c < 4; c++) A.prev_q[i * 4 + c] = A.q[i * 4 + c];
        if (!(A.mtype[i] == 2 && A.awake[i])) continue;
        const double dt = A.w_dt[w];
        const double *g = &A.w_g[w * 3];
        double *v = &A.v[i * 3], *om = &A.w[i * 3];
        const double gf = A.gf[i];
        double v0 = v[0] + (g[0] * gf) * dt, v1 = v[1] + (g[1] * gf) * dt, v2 = v[2] + (g[2] * gf) * dt;
        const double ldmp = A.ld[i] + A.w_def_damp[w * 2];
        const double admp = A.ad[i] + A.w_def_damp[w * 2 + 1];
        const double fl = np_max(1.0 - ldmp * dt, 0.0);
        v0 = v0 * fl; v1 = v1 * fl; v2 = v2 * fl;
        const double speed = sqrt((v0 * v0 + v1 * v1) + v2 * v2);
        const double qs = A.qd[i] * speed;
        v0 = v0 - (qs * v0) * dt; v1 = v1 - (qs * v1) * dt; v2 = v2 - (qs * v2) * dt;
        v[0] = v0; v[1] = v1; v[2] = v2;
        const double fa = np_max(1.0 - admp * dt, 0.0);
        om[0] = om[0] * fa; om[1] = om[1] * fa; om[2] = om[2] * fa;
    }
}

// ---------------------------------------------------------------------------
// narrowphase (narrowphase.py:78-100): one thread per solid pair for the
// analytic routes; convex pairs are queued for the GJK/EPA kernel. Results go
// to a per-pair slot so contact order follows pair order.
// ---------------------------------------------------------------------------
__global__ void k_narrow(Arena A) {
    if (pairs_over(A)) return;
    const int P = A.pair_scan[A.NB];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        int cnt = 0;
        if (A.pair_solid[p]) {
            const int a = A.pair_a[p], b = A.pair_b[p];
            const int ka = A.kind[a], kb = A.kind[b];
            double *s = &A.slot[(size_t)p * SLOT];
            if (ka == 3 || kb == 3) {
                const int idx = atomicAdd(A.gjk_n, 1);
                A.gjk_list[idx] = p;
            } else {
                double nrm[3], pts[12], dep[4];
                const double *pa = &A.pos[a * 3], *pb = &A.pos[b * 3];
                const double *ha = &A.half[a * 3], *hb = &A.half[b * 3];
                double Ra[9], Rb[9];
                quat_to_matrix(&A.q[a * 4], Ra);
                quat_to_matrix(&A.q[b * 4], Rb);
                if (ka == 2 && kb == 2) {
                    cnt = box_box(pa, Ra, ha, pb, Rb, hb, nrm, pts, dep);
                } else if (ka == 1 && kb == 1) {
                    cnt = sphere_sphere(pa, ha[0], pb, hb[0], nrm, pts, dep);
                } else if (ka == 1 && kb == 2) {
                    cnt = sphere_box(pa, ha[0], pb, Rb, hb, nrm, pts, dep);
                } else if (ka == 2 && kb == 1) {
                    cnt = sphere_box(pb, hb[0], pa, Ra, ha, nrm, pts, dep);
                    nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
                }
                if (cnt) {
                    s[0] = nrm[0]; s[1] = nrm[1]; s[2] = nrm[2];
                    for (int j = 0; j < cnt; j++) {
                        s[3 + j * 4] = pts[j * 3]; s[4 + j * 4] = pts[j * 3 + 1];
                        s[5 + j * 4] = pts[j * 3 + 2]; s[6 + j * 4] = dep[j];
                    }
                }
            }
        }
        A.slot_cnt[p] = cnt;
    }
}

__device__ inline void make_proxy(const Arena &A, int i, Proxy &P) {
    const int s = A.shape[i];
    P.kind = A.shape_type[s];
    quat_to_matrix(&A.q[i * 4], P.R);
    for (int c = 0; c < 3; c++) P.c[c] = A.pos[i * 3 + c];
    P.r = A.shape_radius[s];
    for (int c = 0; c < 3; c++) P.h[c] = 0.5 * A.shape_size[s * 3 + c];
    P.local = &A.points[A.pt_off[s] * 3];
    P.m = A.pt_cnt[s];
}

// gjk.collide_convex (gjk.py:249-264) through collide.collide (collide.py:251-269)
__global__ void k_gjk(Arena A) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (pairs_over(A)) return;
    EpaWork &W = reinterpret_cast<EpaWork *>(smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int nitems = *A.gjk_n;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) A.status[ST_GJK_ITEMS] = nitems;
    for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nitems; it += nwarps) {
        const int p = A.gjk_list[it];
        const int a = A.pair_a[p], b = A.pair_b[p];
        Proxy PA, PB;
        make_proxy(A, a, PA);
        make_proxy(A, b, PB);
        double nrm[3], pt[3], dep = 0.0;
        const int r = collide_convex(PA, PB, W, nrm, pt, &dep);
        if (lane == 0) {
            if (r < 0) atomicAdd(&A.status[ST_EPA_LIMIT], 1);
            double *s = &A.slot[(size_t)p * SLOT];
            if (r > 0) {
                s[0] = nrm[0]; s[1] = nrm[1]; s[2] = nrm[2];
                s[3] = pt[0]; s[4] = pt[1]; s[5] = pt[2]; s[6] = dep;
            }
            A.slot_cnt[p] = r > 0 ? 1 : 0;
        }
        __syncwarp();
    }
}

__global__ void k_contact_compact(Arena A) {
    if (overflowed(A)) return;
    const int P = A.pair_scan[A.NB];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const int cnt = A.slot_cnt[p];
        if (!cnt) continue;
        const int base = A.contact_scan[p];
        const double *s = &A.slot[(size_t)p * SLOT];
        for (int j = 0; j < cnt; j++) {
            const int k = base + j;
            A.c_a[k] = A.pair_a[p];
            A.c_b[k] = A.pair_b[p];
            for (int c = 0; c < 3; c++) {
                A.c_n[k * 3 + c] = s[c];
                A.c_pt[k * 3 + c] = s[3 + j * 4 + c];
            }
            A.c_depth[k] = s[6 + j * 4];
            A.c_imp[k * 3] = A.c_imp[k * 3 + 1] = A.c_imp[k * 3 + 2] = 0.0;
        }
    }
}

// contact range of world w in the compacted contact arrays
__device__ __forceinline__ void world_contacts(const Arena &A, int w, int &c0, int &c1) {
    const int p0 = A.pair_scan[A.w_body_off[w]], p1 = A.pair_scan[A.w_body_off[w + 1]];
    c0 = A.contact_scan[p0];
    c1 = A.contact_scan[p1];
}

// ---------------------------------------------------------------------------
// dependency levels for exact Gauss-Seidel order. Constraint k's level is one
// more than the highest level of any earlier constraint sharing a dynamic
// body with it; constraints of one level touch disjoint dynamic bodies, so
// running the levels in order, each level in parallel, reproduces the
// reference's one-at-a-time sweep bit for bit (static and kinematic bodies
// are never written: their inverse mass and inertia are zero).
// Computed by one warp, 32 constraints per batch.
// ---------------------------------------------------------------------------
__device__ inline int warp_levels(int n, const int *ea, const int *eb, const int *mtype,
                                  int *last, int *level) {
    const int lane = threadIdx.x & 31;
    int maxl = -1;
    for (int base = 0; base < n; base += 32) {
        const int k = base + lane;
        const bool valid = k < n;
        const int a = valid ? ea[k] : -1, b = valid ? eb[k] : -1;
        const bool da = a >= 0 && mtype[a] == 2, db = b >= 0 && mtype[b] == 2;
        int lvl = 0;
        if (da) lvl = max(lvl, ((volatile int *)last)[a] + 1);
        if (db) lvl = max(lvl, ((volatile int *)last)[b] + 1);
        unsigned conflict = 0;
        for (int j = 0; j < 32; j++) {
            const int aj = __shfl_sync(FULL, a, j), bj = __shfl_sync(FULL, b, j);
            const bool c = j < lane && ((da && (a == aj || a == bj)) || (db && (b == aj || b == bj)));
            conflict |= (c ? 1u : 0u) << j;
        }
        for (int j = 0; j < 32; j++) {
            const int lj = __shfl_sync(FULL, lvl, j);
            if ((conflict >> j) & 1u) lvl = max(lvl, lj + 1);
        }
        if (valid) {
            level[k] = lvl;
            if (da) atomicMax(&last[a], lvl);
            if (db) atomicMax(&last[b], lvl);
            maxl = max(maxl, lvl);
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) maxl = max(maxl, __shfl_xor_sync(FULL, maxl, o));
    return maxl + 1;
}

// bucket constraints by level: ls[0..D] = level starts, order = constraint ids
__device__ inline void bucket_levels(int n, int D, const int *level, int *ls, int *cursor,
                                     int *order) {
    for (int l = threadIdx.x; l <= D; l += blockDim.x) { ls[l] = 0; cursor[l] = 0; }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) atomicAdd(&ls[level[k] + 1], 1);
    __syncthreads();
    if (threadIdx.x == 0)
        for (int l = 1; l <= D; l++) ls[l] += ls[l - 1];
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int l = level[k];
        order[ls[l] + atomicAdd(&cursor[l], 1)] = k;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// contact solver (solver.py:192-337 with _solver_native.prepare_and_solve,
// _solver_native.pyx:132-312), one CTA per world
// ---------------------------------------------------------------------------
__device__ __forceinline__ double combine(double a, double b, int mode) {
    if (mode == 1) return b < a ? b : a;
    if (mode == 2) return b > a ? b : a;
    if (mode == 3) return a * b;
    return 0.5 * (a + b);
}

__device__ __forceinline__ void material(const Arena &A, int i, double &dynf, double &rest,
                                         int &fc, int &rc) {
    const int m = A.material[i];
    if (m >= 0) { dynf = A.mat_dynf[m]; rest = A.mat_rest[m]; fc = A.mat_fcomb[m]; rc = A.mat_rcomb[m]; }
    else { dynf = 0.6; rest = 0.0; fc = 0; rc = 0; }   // model.DEFAULT_MATERIAL
}

__device__ __forceinline__ unsigned long long pair_key(int a, int b) {
    return ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
}
__device__ __forceinline__ int hash_slot(unsigned long long key, int mask) {
    return (int)((key * 0x9E3779B97F4A7C15ull) >> 40) & mask;
}

__device__ __forceinline__ void rel_vel(const double *lv, const double *av, int a, int b,
                                        const double *rA, const double *rB, double &x, double &y,
                                        double &z) {
    x = (lv[b * 3] + av[b * 3 + 1] * rB[2] - av[b * 3 + 2] * rB[1]) -
        (lv[a * 3] + av[a * 3 + 1] * rA[2] - av[a * 3 + 2] * rA[1]);
    y = (lv[b * 3 + 1] + av[b * 3 + 2] * rB[0] - av[b * 3] * rB[2]) -
        (lv[a * 3 + 1] + av[a * 3 + 2] * rA[0] - av[a * 3] * rA[2]);
    z = (lv[b * 3 + 2] + av[b * 3] * rB[1] - av[b * 3 + 1] * rB[0]) -
        (lv[a * 3 + 2] + av[a * 3] * rA[1] - av[a * 3 + 1] * rA[0]);
}

// _apply_w (_solver_native.pyx:132-151); only dynamic bodies are written
__device__ __forceinline__ void apply_impulse(const Arena &A, double *lv, double *av, int a, int b,
                                              double ima, double imb, const double *rA,
                                              const double *rB, double Px, double Py, double Pz) {
    if (A.mtype[a] == 2) {
        const double *I = &A.invIw[a * 9];
        lv[a * 3] -= ima * Px; lv[a * 3 + 1] -= ima * Py; lv[a * 3 + 2] -= ima * Pz;
        const double cx = rA[1] * Pz - rA[2] * Py, cy = rA[2] * Px - rA[0] * Pz, cz = rA[0] * Py - rA[1] * Px;
        av[a * 3] -= I[0] * cx + I[1] * cy + I[2] * cz;
        av[a * 3 + 1] -= I[3] * cx + I[4] * cy + I[5] * cz;
        av[a * 3 + 2] -= I[6] * cx + I[7] * cy + I[8] * cz;
    }
    if (A.mtype[b] == 2) {
        const double *I = &A.invIw[b * 9];
        lv[b * 3] += imb * Px; lv[b * 3 + 1] += imb * Py; lv[b * 3 + 2] += imb * Pz;
        const double cx = rB[1] * Pz - rB[2] * Py, cy = rB[2] * Px - rB[0] * Pz, cz = rB[0] * Py - rB[1] * Px;
        av[b * 3] += I[0] * cx + I[1] * cy + I[2] * cz;
        av[b * 3 + 1] += I[3] * cx + I[4] * cy + I[5] * cz;
        av[b * 3 + 2] += I[6] * cx + I[7] * cy + I[8] * cz;
    }
}

// _effmass (_solver_native.pyx:154-176)
__device__ __forceinline__ double effmass(const Arena &A, const double *ra, const double *rb,
                                          double dx, double dy, double dz, int a, int b,
                                          double ima, double imb) {
    const double ax = ra[1] * dz - ra[2] * dy, ay = ra[2] * dx - ra[0] * dz, az = ra[0] * dy - ra[1] * dx;
    const double bx = rb[1] * dz - rb[2] * dy, by = rb[2] * dx - rb[0] * dz, bz = rb[0] * dy - rb[1] * dx;
    const double *Ia = &A.invIw[a * 9], *Ib = &A.invIw[b * 9];
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

__device__ inline void wake_body(const Arena &A, int i) {
    A.awake[i] = 1;
    A.timer[i] = 0.0;
}

__device__ __forceinline__ double speed2(const double *v) {
    return (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
}

// contact prep: material combine, warm-start seed, arms, basis, masses, bias
__device__ inline void prep_contact(const Arena &A, int w, int k, bool warm, int cur) {
    const int a = A.c_a[k], b = A.c_b[k];
    double fa, ra_, fb, rb_;
    int fca, rca, fcb, rcb;
    material(A, a, fa, ra_, fca, rca);
    material(A, b, fb, rb_, fcb, rcb);
    const double rest = combine(ra_, rb_, rca);
    double fric = combine(fa, fb, fca);
    {   // pair friction override (world.py:220-223), per-world sorted table
        const int ma = A.material_key[a], mb = A.material_key[b];
        const int ka = ma <= mb ? ma : mb, kb = ma <= mb ? mb : ma;
        int lo = A.w_pf_off[w], hi = lo + A.w_pf_n[w];
        while (lo < hi) {
            int m = (lo + hi) >> 1;
            if (A.pf_a[m] < ka || (A.pf_a[m] == ka && A.pf_b[m] < kb)) lo = m + 1; else hi = m;
        }
        if (lo < A.w_pf_off[w] + A.w_pf_n[w] && A.pf_a[lo] == ka && A.pf_b[lo] == kb) fric = A.pf_mu[lo];
    }
    const double *pt = &A.c_pt[k * 3];
    double n0 = 0.0, t0 = 0.0, t1v = 0.0;
    if (warm) {   // _seed_pair (solver.py:222-233)
        const unsigned long long key = pair_key(a, b);
        int s = hash_slot(key, A.hash_mask);
        const unsigned long long *hk = A.hkey[cur];
        for (int probe = 0; probe <= A.hash_mask; probe++) {
            const unsigned long long kk = hk[s];
            if (kk == ~0ull) break;
            if (kk == key) {
                const int start = A.hval[cur][s * 2], cnt = A.hval[cur][s * 2 + 1];
                double best_d = 0.04;
                for (int e = start; e < start + cnt; e++) {
                    const double *cp = &A.cache_pt[cur][e * 3];
                    const double d0 = pt[0] - cp[0], d1 = pt[1] - cp[1], d2 = pt[2] - cp[2];
                    const double d = d0 * d0 + d1 * d1 + d2 * d2;
                    if (d < best_d) {
                        best_d = d;
                        n0 = A.cache_imp[cur][e * 3];
                        t0 = A.cache_imp[cur][e * 3 + 1];
                        t1v = A.cache_imp[cur][e * 3 + 2];
                    }
                }
                break;
            }
            s = (s + 1) & A.hash_mask;
        }
    }
    A.c_imp[k * 3] = n0; A.c_imp[k * 3 + 1] = t0; A.c_imp[k * 3 + 2] = t1v;
    double *D = &A.c_data[(size_t)k * CD];
    const double ima = A.inv_mass[a], imb = A.inv_mass[b];
    double rA[3], rB[3];
    for (int c = 0; c < 3; c++) { rA[c] = pt[c] - A.pos[a * 3 + c]; rB[c] = pt[c] - A.pos[b * 3 + c]; }
    const double nx = A.c_n[k * 3], ny = A.c_n[k * 3 + 1], nz = A.c_n[k * 3 + 2];
    double axx = 1.0, ayy = 0.0, azz = 0.0;
    if (!((nx >= 0 ? nx : -nx) < 0.9)) { axx = 0.0; ayy = 1.0; }
    double t1x = ayy * nz - azz * ny, t1y = azz * nx - axx * nz, t1z = axx * ny - ayy * nx;
    const double ln = sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
    const double inv = ln > 1e-12 ? 1.0 / ln : 0.0;
    t1x *= inv; t1y *= inv; t1z *= inv;
    const double t2x = ny * t1z - nz * t1y, t2y = nz * t1x - nx * t1z, t2z = nx * t1y - ny * t1x;
    D[0] = rA[0]; D[1] = rA[1]; D[2] = rA[2];
    D[3] = rB[0]; D[4] = rB[1]; D[5] = rB[2];
    D[6] = nx; D[7] = ny; D[8] = nz;
    D[9] = t1x; D[10] = t1y; D[11] = t1z;
    D[12] = t2x; D[13] = t2y; D[14] = t2z;
    D[15] = effmass(A, rA, rB, nx, ny, nz, a, b, ima, imb);
    D[16] = effmass(A, rA, rB, t1x, t1y, t1z, a, b, ima, imb);
    D[17] = effmass(A, rA, rB, t2x, t2y, t2z, a, b, ima, imb);
    double dvx, dvy, dvz;
    rel_vel(A.v, A.w, a, b, rA, rB, dvx, dvy, dvz);
    const double vn0 = dvx * nx + dvy * ny + dvz * nz;
    D[18] = vn0 < -A.w_solver[w * 2] ? -rest * vn0 : 0.0;
    D[19] = fric;
    D[20] = ima;
    D[21] = imb;
}

__device__ inline void warm_contact(const Arena &A, int k) {
    const int a = A.c_a[k], b = A.c_b[k];
    const double *D = &A.c_data[(size_t)k * CD];
    const double n = A.c_imp[k * 3], t0 = A.c_imp[k * 3 + 1], t1 = A.c_imp[k * 3 + 2];
    apply_impulse(A, A.v, A.w, a, b, D[20], D[21], &D[0], &D[3],
                  n * D[6] + t0 * D[9] + t1 * D[12],
                  n * D[7] + t0 * D[10] + t1 * D[13],
                  n * D[8] + t0 * D[11] + t1 * D[14]);
}

// one velocity-iteration update of contact k (_solver_native.pyx:259-295)
__device__ inline void solve_contact(const Arena &A, int k) {
    const int a = A.c_a[k], b = A.c_b[k];
    const double *D = &A.c_data[(size_t)k * CD];
    double *lv = A.v, *av = A.w;
    const double *rA = &D[0], *rB = &D[3];
    const double nx = D[6], ny = D[7], nz = D[8];
    const double ima = D[20], imb = D[21];
    double *imp = &A.c_imp[k * 3];
    double dvx, dvy, dvz;
    rel_vel(lv, av, a, b, rA, rB, dvx, dvy, dvz);
    const double vn = dvx * nx + dvy * ny + dvz * nz;
    double nw = imp[0] - D[15] * (vn - D[18]);
    if (nw < 0.0) nw = 0.0;
    double dL = nw - imp[0];
    imp[0] = nw;
    apply_impulse(A, lv, av, a, b, ima, imb, rA, rB, dL * nx, dL * ny, dL * nz);
    const double maxf = D[19] * nw;
    rel_vel(lv, av, a, b, rA, rB, dvx, dvy, dvz);
    double vt = dvx * D[9] + dvy * D[10] + dvz * D[11];
    double nt = imp[1] - D[16] * vt;
    if (nt > maxf) nt = maxf; else if (nt < -maxf) nt = -maxf;
    dL = nt - imp[1];
    imp[1] = nt;
    apply_impulse(A, lv, av, a, b, ima, imb, rA, rB, dL * D[9], dL * D[10], dL * D[11]);
    vt = dvx * D[12] + dvy * D[13] + dvz * D[14];
    nt = imp[2] - D[17] * vt;
    if (nt > maxf) nt = maxf; else if (nt < -maxf) nt = -maxf;
    dL = nt - imp[2];
    imp[2] = nt;
    apply_impulse(A, lv, av, a, b, ima, imb, rA, rB, dL * D[12], dL * D[13], dL * D[14]);
}

// split-impulse position pass (_solver_native.pyx:297-312)
__device__ inline void position_contact(const Arena &A, int k, double slop) {
    const double vn = A.c_depth[k] - slop;
    if (vn <= 0.0) return;
    const double *D = &A.c_data[(size_t)k * CD];
    const double ima = D[20], imb = D[21];
    if (ima + imb <= 1e-12) return;
    const double dL = 0.8 * vn / (ima + imb);
    const int a = A.c_a[k], b = A.c_b[k];
    if (A.mtype[a] == 2)
        for (int c = 0; c < 3; c++) A.pos[a * 3 + c] -= ima * dL * D[6 + c];
    if (A.mtype[b] == 2)
        for (int c = 0; c < 3; c++) A.pos[b * 3 + c] += imb * dL * D[6 + c];
}

__global__ void k_solve(Arena A) {
    __shared__ int s_flag, s_D;
    if (overflowed(A)) return;
    const int cur = *A.parity;
    for (int w = blockIdx.x; w < A.W; w += gridDim.x) {
        if (!world_collides(A, w)) continue;
        int c0, c1;
        world_contacts(A, w, c0, c1);
        const int K = c1 - c0;
        if (K == 0) continue;                       // solver.py:197-198
        const bool warm = (A.w_flags[w] & WF_WARM) != 0;
        const double thr = 0.15 * 0.15;
        // ---- _wake_sleepers (solver.py:321-337)
        if (threadIdx.x == 0) s_flag = 0;
        __syncthreads();
        for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
            const int e[2] = {A.c_a[k], A.c_b[k]};
            for (int j = 0; j < 2; j++) {
                const int x = e[j];
                if (A.mtype[x] == 2 && !A.awake[x] && speed2(&A.v[x * 3]) > thr) s_flag = 1;
            }
        }
        __syncthreads();
        if (s_flag) {
            // a body asleep at the start could wake and then wake others:
            // resolve in the reference's sequential contact order
            if (threadIdx.x == 0) {
                atomicAdd(&A.status[ST_CASCADE], 1);
                for (int k = c0; k < c1; k++) {
                    const int a = A.c_a[k], b = A.c_b[k];
                    if (!A.awake[b]) {
                        const int t = A.mtype[a];
                        if (t == 1 || (t == 2 && A.awake[a] && speed2(&A.v[a * 3]) > thr)) wake_body(A, b);
                    }
                    if (!A.awake[a]) {
                        const int t = A.mtype[b];
                        if (t == 1 || (t == 2 && A.awake[b] && speed2(&A.v[b * 3]) > thr)) wake_body(A, a);
                    }
                }
            }
        } else {
            // no woken body can wake another: order does not matter
            for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
                const int a = A.c_a[k], b = A.c_b[k];
                const int ta = A.mtype[a], tb = A.mtype[b];
                if (!A.awake[b] && (ta == 1 || (ta == 2 && A.awake[a] && speed2(&A.v[a * 3]) > thr)))
                    wake_body(A, b);
                if (!A.awake[a] && (tb == 1 || (tb == 2 && A.awake[b] && speed2(&A.v[b * 3]) > thr)))
                    wake_body(A, a);
            }
        }
        __syncthreads();
        // ---- per-contact prep (parallel; reads velocities before any impulse)
        for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x) prep_contact(A, w, k, warm, cur);
        const int b0 = A.w_body_off[w], b1 = b0 + A.w_body_n[w];
        for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) A.b_last[i] = -1;
        __syncthreads();
        // ---- Gauss-Seidel levels
        if (threadIdx.x < 32) {
            const int D = warp_levels(K, A.c_a + c0, A.c_b + c0, A.mtype, A.b_last, A.c_level + c0);
            if (threadIdx.x == 0) s_D = D;
        }
        __syncthreads();
        const int D = s_D;
        int *ls = A.c_level_start + c0 + w;
        int *cursor = A.c_level_start + (A.contact_cap + A.W + 1) + c0 + w;
        int *order = A.c_order + c0;
        bucket_levels(K, D, A.c_level + c0, ls, cursor, order);
        // ---- warm start, iterations, position pass, level by level
        if (warm) {
            for (int l = 0; l < D; l++) {
                for (int j = ls[l] + threadIdx.x; j < ls[l + 1]; j += blockDim.x) warm_contact(A, c0 + order[j]);
                __syncthreads();
            }
        }
        const int iters = A.w_iters[w];
        for (int it = 0; it < iters; it++) {
            for (int l = 0; l < D; l++) {
                for (int j = ls[l] + threadIdx.x; j < ls[l + 1]; j += blockDim.x) solve_contact(A, c0 + order[j]);
                __syncthreads();
            }
        }
        const double slop = A.w_solver[w * 2 + 1];
        for (int l = 0; l < D; l++) {
            for (int j = ls[l] + threadIdx.x; j < ls[l + 1]; j += blockDim.x) position_contact(A, c0 + order[j], slop);
            __syncthreads();
        }
    }
}

}  // namespace omi
