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
#include <cooperative_groups.h>

#include "arena.cuh"
#include "geometry.cuh"
#include "gjk.cuh"
#include "capsule.cuh"

namespace omi {

constexpr int WF_SLEEP = 1, WF_WARM = 2, WF_COLLISION = 4;
constexpr unsigned FULL = 0xffffffffu;

// a slot of a work list whose order does not matter: the lanes that reach
// this call together take consecutive slots with one increment of the list's
// counter (one increment per lane serialises every list entry of a launch on
// one address)
__device__ __forceinline__ int list_slot(int *counter) {
    cooperative_groups::coalesced_group g = cooperative_groups::coalesced_threads();
    int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(counter, (int)g.size());
    return g.shfl(base, 0) + (int)g.thread_rank();
}

__device__ __forceinline__ bool pairs_over(const Arena &A) {
    return A.pair_scan[A.NB] > A.pair_cap;
}
// pair or contact overflow, or a sweep wait that ran out earlier in this
// launch of steps: the rest of the step (and every later step of the launch)
// does nothing; valid once the contact scan of this step ran
__device__ __forceinline__ bool overflowed(const Arena &A) {
    if (A.pair_scan[A.NB] > A.pair_cap) return true;
    if (A.contact_scan[A.pair_scan[A.NB]] > A.contact_cap) return true;
    return *(volatile const int *)&A.status[ST_SWEEP_TIMEOUT] != 0;
}
__device__ __forceinline__ bool world_collides(const Arena &A, int w) {
    return A.w_active[w] && (A.w_flags[w] & WF_COLLISION);
}
// a world whose sort, levels, wake, sweep, cache store and sleep pass run on
// many blocks (wide.cuh); the one-block-per-world kernels skip it
__device__ __forceinline__ bool world_wide(const Arena &A, int w) { return A.w_wide[w] != 0; }
__device__ __forceinline__ bool dyn(const Arena &A, int i) { return A.mtype[i] == 2; }

// ---------------------------------------------------------------------------
// refit: world AABBs (world.py:471-508) and world inverse inertia
// einsum('nij,nkj->nik', R*invI, R) (solver.py:215-220), one thread per body
// ---------------------------------------------------------------------------
__global__ void k_refit(Arena A) {
    if (blockIdx.x == 0 && threadIdx.x == 0) { A.gjk_n[0] = 0; A.clip_n[0] = 0; A.trig_n[0] = 0; A.mesh_n[0] = 0; }
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
        } else if (kind == 3 || kind == 5) {         // hull or mesh: world points min / max
            const int s = A.rshape[i];
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
        } else if (kind == 4) {
            // CapsuleProxy.aabb (body.py:84-98): segment ends min/max -+ radius
            double e0[3], e1[3];
            capsule_ends(p, R, h[1], e0, e1);
            for (int c = 0; c < 3; c++) {
                lo[c] = ((e0[c] < e1[c] ? e0[c] : e1[c]) - h[0]) - 0.05;
                hi[c] = ((e0[c] > e1[c] ? e0[c] : e1[c]) + h[0]) + 0.05;
            }
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
// numpy's sort order: NaN after every number (+inf included), NaNs among
// themselves (and equal keys) by index
__device__ __forceinline__ bool key_less(double ka, int va, double kb, int vb) {
    const bool na = ka != ka, nb = kb != kb;
    if (na | nb) return na == nb ? va < vb : nb;
    return ka < kb || (!(kb < ka) && va < vb);
}

// ROWS: also write each sorted row's box (the step's broadphase reads them)
template <bool ROWS>
__global__ void k_sort(Arena A, int smem_cap) {
    extern __shared__ __align__(16) unsigned char smem[];
    for (int w = blockIdx.x; w < A.W; w += gridDim.x) {
        if (!world_collides(A, w) || (ROWS && world_wide(A, w))) continue;
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
            k0[i] = A.aabb_min[(off + i) * 3] + 0.0;    // -0.0 == 0.0; NaN stays NaN (sorts last)
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
            const int body = off + v0[i];
            A.order[off + i] = body;
            A.sorted_x[off + i] = k0[i];
            if (!ROWS) continue;
            // the row's box in sorted order, so the sweep windows read rows contiguously
            double4 *row = reinterpret_cast<double4 *>(&A.srt_box[(size_t)(off + i) * 8]);
            const double *lo = &A.aabb_min[body * 3], *hi = &A.aabb_max[body * 3];
            row[0] = make_double4(lo[0], hi[0], lo[1], hi[1]);
            row[1] = make_double4(lo[2], hi[2], 0.0, 0.0);
            const bool sensor = A.tshape[body] >= 0;
            A.srt_info[off + i] = A.mtype[body] | (A.shape[body] >= 0 && !sensor ? 4 : 0) |
                                  (A.awake[body] ? 8 : 0) | (sensor ? 16 : 0) | (A.filter_row[body] << 5);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// sweep-and-prune windows (broadphase.py:262-294): for sorted row k the
// candidates are rows k+1 .. searchsorted(lo_sx, hi_sx[k], 'right')-1; keep
// y/z overlap (>=), at least one dynamic body and interacting filters. One
// warp per sorted row; lanes test 32 candidates at a time and a ballot keeps
// the reference's k-major, then kj, order. The step's kernels read the rows'
// boxes in sorted order (written by k_sort); the count pass records each
// window's end and which of its first 64 rows it kept, so the emit pass
// tests only rows past those 64. The helpers below serve the allocation-free
// entry point, which reads the caller's boxes in place.
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

// (numpy's searchsorted order: a NaN row is past every finite bound, and a
// NaN bound is past every row)
__device__ __forceinline__ int window_end(const Arena &A, int off, int end_w, double hx) {
    if (hx != hx) return end_w;
    int lo = off, hi = end_w;
    while (lo < hi) {
        int m = (lo + hi) >> 1;
        if (A.sorted_x[m] <= hx) lo = m + 1; else hi = m;
    }
    return lo;
}

// the count pass on boxes read in place (no sorted rows, no recorded window
// ends): the allocation-free entry point's form
__global__ void k_pair_count_boxes(Arena A) {
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


// first row k in [lo, hi) with !(sorted_x[k] <= hx), else hi - the binary
// search above done 32-ary by a warp (one load per lane per step, ~3 steps)
__device__ __forceinline__ int window_end_warp(const double *sx, int lo, int hi, double hx) {
    const int lane = threadIdx.x & 31;
    if (hx != hx) return hi;                         // warp-uniform: one row's bound
    while (hi - lo > 32) {
        const int step = (hi - lo + 31) >> 5;
        const int k = lo + lane * step;
        const bool t = k < hi ? !(sx[k] <= hx) : true;
        const unsigned m = __ballot_sync(FULL, t);
        const int f = m ? __ffs(m) - 1 : 32;
        const int nlo = f > 0 ? lo + (f - 1) * step + 1 : lo;
        const int nhi = f < 32 ? min(hi, lo + f * step) : hi;
        lo = nlo;
        hi = nhi;
    }
    const bool t = lo + lane < hi ? !(sx[lo + lane] <= hx) : true;
    const unsigned m = __ballot_sync(FULL, t);
    return m ? min(hi, lo + __ffs(m) - 1) : hi;      // m == 0: 32 rows left, none past hx
}

// pair_keep on sorted rows: `ra`/`rb` are the rows' boxes (lo/hi x, y, z),
// `ia`/`ib` their info words: motion type (bits 0-1), collider and no sensor
// (2), awake (3), sensor (4), filter row (5-)
__device__ __forceinline__ bool row_keep(const Arena &A, int w, const double4 &a0, const double4 &a1, int ia,
                                         const double4 &b0, const double4 &b1, int ib) {
    bool keep = (a0.w >= b0.z) & (b0.w >= a0.z) & (a1.y >= b1.x) & (b1.y >= a1.x);
    keep &= ((ia & 3) == 2) | ((ib & 3) == 2);
    if (keep) {
        const int rows = A.w_filter_rows[w];
        OMI_BOUNDS(A, ia >> 5, rows, BS_FILTER_ROW, return false)
        OMI_BOUNDS(A, ib >> 5, rows, BS_FILTER_ROW, return false)
        keep = A.filter_matrix[A.w_filter_off[w] + (ia >> 5) * rows + (ib >> 5)] != 0;
    }
    return keep;
}

__global__ void k_pair_count(Arena A) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.NB; e += nwarps) {
        const int w = A.body_world[e];
        int cnt = 0, endk = e + 1;
        unsigned long long kept = 0;
        if (world_collides(A, w) && e - A.w_body_off[w] < A.w_body_n[w]) {
            const int off = A.w_body_off[w], end_w = off + A.w_body_n[w];
            const double4 *ra = reinterpret_cast<const double4 *>(&A.srt_box[(size_t)e * 8]);
            const double4 a0 = ra[0], a1 = ra[1];
            const int ia = A.srt_info[e];
            endk = window_end_warp(A.sorted_x, off, end_w, a0.y);
            for (int base = e + 1, c = 0; base < endk; base += 32, c++) {
                const int kj = base + lane;
                bool keep = false;
                if (kj < endk) {
                    const double4 *rb = reinterpret_cast<const double4 *>(&A.srt_box[(size_t)kj * 8]);
                    keep = row_keep(A, w, a0, a1, ia, rb[0], rb[1], A.srt_info[kj]);
                }
                const unsigned m = __ballot_sync(FULL, keep);
                if (c < 2) kept |= (unsigned long long)m << (32 * c);
                cnt += __popc(m);
            }
        }
        if (lane == 0) { A.pair_cnt[e] = cnt; A.pair_end[e] = endk; A.pair_mask[e] = kept; }
    }
}

__global__ void k_pair_emit(Arena A) {
    if (pairs_over(A)) return;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.NB; e += nwarps) {
        const int w = A.body_world[e];
        if (!world_collides(A, w) || e - A.w_body_off[w] >= A.w_body_n[w]) continue;
        const int endk = A.pair_end[e];
        if (endk <= e + 1) continue;
        const int a = A.order[e];
        const double4 *ra = reinterpret_cast<const double4 *>(&A.srt_box[(size_t)e * 8]);
        const double4 a0 = ra[0], a1 = ra[1];
        const int ia = A.srt_info[e];
        const unsigned long long kept = A.pair_mask[e];
        int out = A.pair_scan[e];
        for (int base = e + 1, c = 0; base < endk; base += 32, c++) {
            const int kj = base + lane;
            int b = -1, ib = 0;
            bool keep = false;
            if (c < 2) {                             // decided by the count pass
                keep = (kept >> (32 * c + lane)) & 1ull;
                if (keep) { ib = A.srt_info[kj]; b = A.order[kj]; }
            } else if (kj < endk) {
                const double4 *rb = reinterpret_cast<const double4 *>(&A.srt_box[(size_t)kj * 8]);
                ib = A.srt_info[kj];
                keep = row_keep(A, w, a0, a1, ia, rb[0], rb[1], ib);
                if (keep) b = A.order[kj];
            }
            const unsigned m = __ballot_sync(FULL, keep);
            if (keep) {
                const int slot = out + __popc(m & ((1u << lane) - 1u));
                A.pair_a[slot] = a < b ? a : b;
                A.pair_b[slot] = a < b ? b : a;
                // solid-pair filter (world.py:663-670): a sensor on either body makes
                // a sensor pair; else both colliders and an awake mover
                const bool ma = ((ia & 3) == 2 && (ia & 8)) || (ia & 3) == 1;
                const bool mb = ((ib & 3) == 2 && (ib & 8)) || (ib & 3) == 1;
                A.pair_solid[slot] = ((ia | ib) & 16) ? 2 : (((ia & 4) && (ib & 4) && (ma || mb)) ? 1 : 0);
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
// resolve_gravity with the world's volumes (world.py:386-396,
// gravity.py:82-108): the world vector, then each volume whose region holds
// the body's position, in application order: replace sets the field, stop
// zeroes, otherwise the field adds. A point field is normalize(centre - pos)
// times its magnitude; a directional field arrives precomputed.
__device__ __forceinline__ void body_gravity(const Arena &A, int w, int i, double *g) {
    g[0] = A.w_g[w * 3]; g[1] = A.w_g[w * 3 + 1]; g[2] = A.w_g[w * 3 + 2];
    const int v1 = A.w_vol_off[w + 1];
    for (int k = A.w_vol_off[w]; k < v1; k++) {
        const int kind = A.vol_kind[k];
        const double *pos = &A.pos[i * 3], *rc = &A.vol_rc[k * 3], *rr = &A.vol_rr[k * 3];
        bool inside = true;
        if (kind & 2) {
            const double d[3] = {pos[0] - rc[0], pos[1] - rc[1], pos[2] - rc[2]};
            inside = dot_blas(d, d) <= rr[0];
        } else if (kind & 4) {
            inside = fabs(pos[0] - rc[0]) <= rr[0] && fabs(pos[1] - rc[1]) <= rr[1] &&
                     fabs(pos[2] - rc[2]) <= rr[2];
        }
        if (!inside) continue;
        if (kind & 16) { g[0] = g[1] = g[2] = 0.0; continue; }
        const double *fd = &A.vol_field[k * 3];
        double f[3];
        if (kind & 1) {
            const double d[3] = {fd[0] - pos[0], fd[1] - pos[1], fd[2] - pos[2]};
            double u[3];
            normalize3(d, u);
            f[0] = u[0] * A.vol_g[k]; f[1] = u[1] * A.vol_g[k]; f[2] = u[2] * A.vol_g[k];
        } else {
            f[0] = fd[0]; f[1] = fd[1]; f[2] = fd[2];
        }
        if (kind & 8) { g[0] = f[0]; g[1] = f[1]; g[2] = f[2]; }
        else { g[0] = g[0] + f[0]; g[1] = g[1] + f[1]; g[2] = g[2] + f[2]; }
    }
}

__global__ void k_integrate_forces(Arena A, int gated) {
    if (gated && overflowed(A)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.NB; i += gridDim.x * blockDim.x) {
        const int w = A.body_world[i];
        if (!A.w_active[w] || i - A.w_body_off[w] >= A.w_body_n[w]) continue;
        for (int c = 0; c < 3; c++) A.prev_pos[i * 3 + c] = A.pos[i * 3 + c];
        for (int c = 0; c < 4; c++) A.prev_q[i * 4 + c] = A.q[i * 4 + c];
        if (!(A.mtype[i] == 2 && A.awake[i])) continue;
        const double dt = A.w_dt[w];
        double g[3];
        body_gravity(A, w, i, g);
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

#ifdef OMI_BOUNDS_CHECK
// Test hook of the bounds-checked build (omi_bounds_probe): the narrowphase
// checks candidate pair g_bounds_probe as if its first body index were past
// the arena, so a test can make a check fail without corrupting anything.
// -1 (the default) is off. One variable per device, for every context there.
__device__ int g_bounds_probe = -1;
__device__ __forceinline__ int bounds_probe(int p, int a, int nb) {
    return p == *(volatile int *)&g_bounds_probe ? nb : a;
}
#endif

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
        const int kindp = A.pair_solid[p];
        if (kindp == 2) {
            A.trig_list[list_slot(A.trig_n)] = p;     // overlap tested after the solve
        } else if (kindp == 1) {
            const int a = A.pair_a[p], b = A.pair_b[p];
            OMI_BOUNDS(A, bounds_probe(p, a, A.NB), A.NB, BS_PAIR_BODY, A.slot_cnt[p] = 0; continue)
            OMI_BOUNDS(A, b, A.NB, BS_PAIR_BODY, A.slot_cnt[p] = 0; continue)
            const int ka = A.kind[a], kb = A.kind[b];
            double *s = &A.slot[(size_t)p * SLOT];
            if (ka == 5 || kb == 5) {
                // the mesh route (collide.py:272-306): counted by k_mesh_count,
                // written straight into the contact arrays by k_mesh_emit
                A.pair_solid[p] = 3;
                A.mesh_list[list_slot(A.mesh_n)] = p;
            } else if (ka >= 3 || kb >= 3) {
                const int idx = list_slot(A.gjk_n);
                A.gjk_list[idx] = p;
            } else {
                double nrm[3], pts[12], dep[4];
                const double *pa = &A.pos[a * 3], *pb = &A.pos[b * 3];
                const double *ha = &A.half[a * 3], *hb = &A.half[b * 3];
                double Ra[9], Rb[9];
                quat_to_matrix(&A.q[a * 4], Ra);
                quat_to_matrix(&A.q[b * 4], Rb);
                if (ka == 2 && kb == 2) {
                    // the six face axes here (they separate most candidate
                    // pairs); the pairs they leave carry their best axis so
                    // far to k_edge_clip, which runs the nine edge axes and
                    // clips the touching ones, in warps of survivors only
                    SatBest best;
                    sat_begin(best);
                    if (sat_axes(0, 6, pa, Ra, ha, pb, Rb, hb, best)) {
                        s[0] = best.x; s[1] = best.y; s[2] = best.z; s[3] = best.depth;
                        A.clip_list[list_slot(A.clip_n)] = p;
                    }
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

// the box-box pairs no face axis separated (k_narrow), one thread per pair:
// the nine edge axes from the best face axis k_narrow left in the slot, then
// face clipping of the touching ones (_collide_native.pyx:20-263) into the
// pair's slot
__global__ void k_edge_clip(Arena A) {
    if (pairs_over(A)) return;
    const int n = *A.clip_n;
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < n; it += gridDim.x * blockDim.x) {
        const int p = A.clip_list[it];
        const int a = A.pair_a[p], b = A.pair_b[p];
        double *s = &A.slot[(size_t)p * SLOT];
        double Ra[9], Rb[9], pts[12], dep[4];
        quat_to_matrix(&A.q[a * 4], Ra);
        quat_to_matrix(&A.q[b * 4], Rb);
        SatBest best;
        best.x = s[0]; best.y = s[1]; best.z = s[2]; best.depth = s[3];
        if (!sat_axes(6, 15, &A.pos[a * 3], Ra, &A.half[a * 3], &A.pos[b * 3], Rb, &A.half[b * 3], best))
            continue;                                   // separated: k_narrow left the count at 0
        double nrm[3] = {best.x, best.y, best.z};
        const double depth = best.depth;
        const int cnt = clip_faces(&A.pos[a * 3], Ra, &A.half[a * 3], &A.pos[b * 3], Rb, &A.half[b * 3], nrm, depth,
                                   pts, dep);
        if (cnt) {
            s[0] = nrm[0]; s[1] = nrm[1]; s[2] = nrm[2];
            for (int j = 0; j < cnt; j++) {
                s[3 + j * 4] = pts[j * 3]; s[4 + j * 4] = pts[j * 3 + 1];
                s[5 + j * 4] = pts[j * 3 + 2]; s[6 + j * 4] = dep[j];
            }
        }
        A.slot_cnt[p] = cnt;
    }
}

// make_proxy (body.py:214-237) of shape s at body i's pose
__device__ inline void make_proxy_shape(const Arena &A, int s, int i, Proxy &P) {
#ifdef OMI_BOUNDS_CHECK
    // a shape or hull point range outside the tables: a point proxy at the
    // body's centre (no table read; the step is reported as failed)
    if (!bounds_ok(A.status, s, A.NS, BS_SHAPE) ||
        (A.pt_cnt[s] > 0 && !bounds_ok(A.status, (long long)A.pt_off[s] + A.pt_cnt[s] - 1, A.NPTS, BS_SHAPE))) {
        P.kind = 1;
        quat_to_matrix(&A.q[i * 4], P.R);
        for (int c = 0; c < 3; c++) { P.c[c] = A.pos[i * 3 + c]; P.h[c] = 0.0; }
        P.r = 0.0;
        P.local = A.points;
        P.m = 0;
        return;
    }
#endif
    P.kind = A.shape_type[s];
    quat_to_matrix(&A.q[i * 4], P.R);
    for (int c = 0; c < 3; c++) P.c[c] = A.pos[i * 3 + c];
    P.r = A.shape_radius[s];
    for (int c = 0; c < 3; c++) P.h[c] = 0.5 * A.shape_size[s * 3 + c];
    P.local = &A.points[A.pt_off[s] * 3];
    P.m = A.pt_cnt[s];
    if (P.kind == 4) capsule_ends(P.c, P.R, 0.5 * A.shape_size[s * 3 + 1], P.e0, P.e1);
}

__device__ inline void make_proxy(const Arena &A, int i, Proxy &P) { make_proxy_shape(A, A.shape[i], i, P); }

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
        const int r = collide_convex(PA, PB, W, nrm, pt, &dep, A.epa_faces);
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

// ---------------------------------------------------------------------------
// sensor overlaps (triggers.py:24-72), after the contact solve as the
// reference's _CollisionStages.run does them (world.py:674-676): one warp per
// sensor pair, len(collide.collide(trigger, other, ...)) > 0 with the sensor
// shape at the sensor body's pose against the other body's collider (else
// its sensor). Sphere routes follow collide.sphere_sphere / sphere_box
// (collide.py:56-88); box-box is non-empty exactly when no separating axis
// exists; every other pair goes through GJK/EPA.
// ---------------------------------------------------------------------------
__device__ inline bool py_sphere_sphere_hit(const Proxy &A, const Proxy &B) {
    const double d[3] = {B.c[0] - A.c[0], B.c[1] - A.c[1], B.c[2] - A.c[2]};
    return !(sqrt(dot_blas(d, d)) >= A.r + B.r);
}

__device__ inline bool py_sphere_box_hit(const Proxy &S, const Proxy &B) {
    const double v[3] = {S.c[0] - B.c[0], S.c[1] - B.c[1], S.c[2] - B.c[2]};
    double delta[3];
    for (int j = 0; j < 3; j++) {
        const double col[3] = {B.R[j], B.R[3 + j], B.R[6 + j]};
        const double l = dot_blas(col, v);
        double cl = l > -B.h[j] ? l : -B.h[j];
        cl = cl < B.h[j] ? cl : B.h[j];
        delta[j] = l - cl;
    }
    return !(sqrt(dot_blas(delta, delta)) > S.r);
}

__global__ void k_triggers(Arena A) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (overflowed(A)) return;
    EpaWork &W = reinterpret_cast<EpaWork *>(smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int nitems = *A.trig_n;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nitems; it += nwarps) {
        const int p = A.trig_list[it];
        const int i = A.pair_a[p], j = A.pair_b[p];
        const int ti = A.tshape[i], tj = A.tshape[j];
        const int trg = ti >= 0 ? i : j, other = ti >= 0 ? j : i;
        const int ts = ti >= 0 ? ti : tj;
        const int os = A.shape[other] >= 0 ? A.shape[other] : A.tshape[other];
        int hit = -1;
        if (os >= 0) {
            Proxy PA, PB;
            make_proxy_shape(A, ts, trg, PA);
            make_proxy_shape(A, os, other, PB);
            if (PA.kind == 1 && PB.kind == 1) {
                hit = py_sphere_sphere_hit(PA, PB);
            } else if (PA.kind == 1 && PB.kind == 2) {
                hit = py_sphere_box_hit(PA, PB);
            } else if (PA.kind == 2 && PB.kind == 1) {
                hit = py_sphere_box_hit(PB, PA);
            } else if (PA.kind == 2 && PB.kind == 2) {
                double nrm[3], depth;
                hit = box_box_sat(PA.c, PA.R, PA.h, PB.c, PB.R, PB.h, nrm, depth) ? 1 : 0;
            } else {
                double nrm[3], pt[3], dep = 0.0;
                const int r = collide_convex(PA, PB, W, nrm, pt, &dep, A.epa_faces);
                if (r < 0 && lane == 0) atomicAdd(&A.status[ST_EPA_LIMIT], 1);
                hit = r > 0 ? 1 : 0;
            }
        }
        if (lane == 0) {
            A.trig_out[it * 3] = trg;
            A.trig_out[it * 3 + 1] = other;
            A.trig_out[it * 3 + 2] = hit;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// triangle meshes (collide.py:272-306 with trigrid.py): a static or kinematic mesh body
// against another body, one warp per pair. The candidates are the triangles
// the reference's uniform grid hands back for the other proxy's bounds
// (trigrid.py:99-111): every triangle whose bounds meet the query when the
// mesh has fewer than 256 triangles, else the oversized ones plus those
// binned in a cell the query's cell range covers. A capsule is tested
// against its candidates in one pass (capsule_triangle_batch), any other
// proxy through GJK/EPA with one candidate triangle at a time. Contacts come
// in ascending triangle order, normals from a to b. k_mesh_count writes the
// pair's count for the contact scan; k_mesh_emit repeats the pass and writes
// the contacts at the pair's place in the contact arrays.
// ---------------------------------------------------------------------------
// A kinematic mesh's tables at this step's pose, one block per mesh: world
// vertices (points @ R.T + position), per-triangle bounds and the uniform
// grid of trigrid.py:63-97 - the reference rebuilds a moving mesh's proxy and
// grid every step (narrowphase.py:40-48). Static meshes keep the tables the
// host built at load.
constexpr int MESH_REFRESH_THREADS = 256;

__global__ void __launch_bounds__(MESH_REFRESH_THREADS) k_mesh_refresh(Arena A, int n_meshes) {
    __shared__ double red[MESH_REFRESH_THREADS];
    __shared__ int redi[MESH_REFRESH_THREADS];
    __shared__ double glo[3], ghi[3];
    __shared__ int shape[3];
    if (pairs_over(A)) return;
    const int tid = threadIdx.x;
    for (int m = blockIdx.x; m < n_meshes; m += gridDim.x) {
        const int mb = A.mesh_body_of[m];
        const int w = A.body_world[mb];
        if (A.mtype[mb] == 0 || !world_collides(A, w)) continue;
        double R[9];
        quat_to_matrix(&A.q[mb * 4], R);
        const double *c = &A.pos[mb * 3];
        const int s = A.rshape[mb];
        const double *pts = &A.points[A.pt_off[s] * 3];
        const int t0 = A.mesh_tri_off[m], t1 = A.mesh_tri_off[m + 1], T = t1 - t0;
        double *tv = const_cast<double *>(A.tri_verts), *tb = const_cast<double *>(A.tri_box);
        double lmin[3] = {INFINITY, INFINITY, INFINITY}, lmax[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int t = t0 + tid; t < t1; t += blockDim.x) {
            double v[9];
            for (int j = 0; j < 3; j++) {
                const double *l = &pts[A.tri_idx[t * 3 + j] * 3];
                for (int k = 0; k < 3; k++) v[j * 3 + k] = dot_blas(l, &R[k * 3]) + c[k];
            }
            for (int k = 0; k < 9; k++) tv[(size_t)t * 9 + k] = v[k];
            for (int k = 0; k < 3; k++) {
                const double a = v[k], b = v[3 + k], d = v[6 + k];
                double mn = a < b ? a : b, mx = a > b ? a : b;
                mn = mn < d ? mn : d;
                mx = mx > d ? mx : d;
                tb[(size_t)t * 6 + k] = mn;
                tb[(size_t)t * 6 + 3 + k] = mx;
                lmin[k] = mn < lmin[k] ? mn : lmin[k];
                lmax[k] = mx > lmax[k] ? mx : lmax[k];
            }
        }
        int *gi = const_cast<int *>(&A.mesh_grid_i[m * 4]);
        double *gd = const_cast<double *>(&A.mesh_grid_d[m * 7]);
        if (T < 256) {                                   // no grid: every query scans exactly
            if (tid == 0) gi[0] = 1;
            __syncthreads();
            continue;
        }
        // lows.min(axis=0), highs.max(axis=0)
        for (int k = 0; k < 3; k++) {
            red[tid] = lmin[k];
            __syncthreads();
            for (int h = blockDim.x / 2; h > 0; h >>= 1) {
                if (tid < h) red[tid] = red[tid + h] < red[tid] ? red[tid + h] : red[tid];
                __syncthreads();
            }
            if (tid == 0) glo[k] = red[0];
            __syncthreads();
            red[tid] = lmax[k];
            __syncthreads();
            for (int h = blockDim.x / 2; h > 0; h >>= 1) {
                if (tid < h) red[tid] = red[tid + h] > red[tid] ? red[tid + h] : red[tid];
                __syncthreads();
            }
            if (tid == 0) ghi[k] = red[0];
            __syncthreads();
        }
        // cell = max(maximum(high - low, 1e-9)) / 64
        double ext = 0.0;
        for (int k = 0; k < 3; k++) {
            double e = ghi[k] - glo[k];
            e = e > 1e-9 ? e : 1e-9;
            ext = k == 0 || e > ext ? e : ext;
        }
        const double cell = ext / 64.0;
        const long long top = (1LL << 30) - 1;
        int lmaxc[3] = {0, 0, 0};
        int *tc = const_cast<int *>(A.tri_cells);
        uint8_t *big = const_cast<uint8_t *>(A.tri_big);
        for (int t = t0 + tid; t < t1; t += blockDim.x) {
            long long f[3], l[3];
            for (int k = 0; k < 3; k++) {
                long long a = (long long)floor((tb[(size_t)t * 6 + k] - glo[k]) / cell);
                long long b = (long long)floor((tb[(size_t)t * 6 + 3 + k] - glo[k]) / cell);
                f[k] = a < 0 ? 0 : (a > top ? top : a);
                l[k] = b < 0 ? 0 : (b > top ? top : b);
                tc[(size_t)t * 6 + k] = (int)f[k];
                tc[(size_t)t * 6 + 3 + k] = (int)l[k];
                lmaxc[k] = (int)l[k] > lmaxc[k] ? (int)l[k] : lmaxc[k];
            }
            big[t] = (l[0] - f[0] + 1) * (l[1] - f[1] + 1) * (l[2] - f[2] + 1) > 64 ? 1 : 0;
        }
        for (int k = 0; k < 3; k++) {
            redi[tid] = lmaxc[k];
            __syncthreads();
            for (int h = blockDim.x / 2; h > 0; h >>= 1) {
                if (tid < h) redi[tid] = redi[tid + h] > redi[tid] ? redi[tid + h] : redi[tid];
                __syncthreads();
            }
            if (tid == 0) shape[k] = redi[0] + 1;
            __syncthreads();
        }
        if (tid == 0) {
            gi[0] = 0; gi[1] = shape[0]; gi[2] = shape[1]; gi[3] = shape[2];
            gd[0] = glo[0]; gd[1] = glo[1]; gd[2] = glo[2];
            gd[3] = ghi[0]; gd[4] = ghi[1]; gd[5] = ghi[2]; gd[6] = cell;
        }
        __syncthreads();
    }
}

// the proxy's own bounds, no margin (body.py: aabb() of each proxy kind)
__device__ inline void proxy_bounds(const Proxy &P, double *lo, double *hi) {
    if (P.kind == 1) {
        for (int c = 0; c < 3; c++) { lo[c] = P.c[c] - P.r; hi[c] = P.c[c] + P.r; }
    } else if (P.kind == 2) {              // _box_corners(half) @ R.T + center
        for (int c = 0; c < 3; c++) { lo[c] = INFINITY; hi[c] = -INFINITY; }
        for (int k = 0; k < 8; k++) {
            const double sv[3] = {(k & 4) ? P.h[0] : -P.h[0], (k & 2) ? P.h[1] : -P.h[1], (k & 1) ? P.h[2] : -P.h[2]};
            for (int c = 0; c < 3; c++) {
                const double x = dot_blas(sv, &P.R[c * 3]) + P.c[c];
                lo[c] = x < lo[c] ? x : lo[c];
                hi[c] = x > hi[c] ? x : hi[c];
            }
        }
    } else if (P.kind == 4) {
        for (int c = 0; c < 3; c++) {
            lo[c] = (P.e0[c] < P.e1[c] ? P.e0[c] : P.e1[c]) - P.r;
            hi[c] = (P.e0[c] > P.e1[c] ? P.e0[c] : P.e1[c]) + P.r;
        }
    } else {
        for (int i = 0; i < P.m; i++)
            for (int c = 0; c < 3; c++) {
                const double x = dot_blas(&P.local[i * 3], &P.R[c * 3]) + P.c[c];
                if (i == 0 || x < lo[c]) lo[c] = x;
                if (i == 0 || x > hi[c]) hi[c] = x;
            }
    }
}

// numpy's float floor division (npy_divmod): fmod, then snap to the integer
__device__ inline double py_floordiv(double a, double b) {
    double mod = fmod(a, b);
    double div = (a - mod) / b;
    if (mod != 0.0 && ((b < 0) != (mod < 0))) div -= 1.0;
    if (div != 0.0) {
        double fd = floor(div);
        if (div - fd > 0.5) fd += 1.0;
        return fd;
    }
    return copysign(0.0, a / b);
}

// TriangleGrid._corner (trigrid.py:113-127) on one axis
__device__ inline int grid_corner(double p, double low, double cell, int shape) {
    const double q = py_floordiv(p - low, cell);
    long long c = (long long)q;
    c = c < 0 ? 0 : c;
    return (int)(c > shape - 1 ? shape - 1 : c);
}

__device__ int mesh_pair(const Arena &A, int p, bool emit, EpaWork &W) {
    const int lane = threadIdx.x & 31;
    const int a = A.pair_a[p], b = A.pair_b[p];
    const bool mesh_is_a = A.kind[a] == 5;
    const int mb = mesh_is_a ? a : b, ob = mesh_is_a ? b : a;
    const int m = A.body_mesh[mb];
    Proxy O;
    make_proxy(A, ob, O);
    double lo[3], hi[3];
    proxy_bounds(O, lo, hi);
    const int *gi = &A.mesh_grid_i[m * 4];
    const double *gd = &A.mesh_grid_d[m * 7];
    const bool exact = gi[0] != 0;
    bool outside = false;
    int fq[3] = {0, 0, 0}, lq[3] = {0, 0, 0};
    if (!exact) {
        for (int k = 0; k < 3; k++) outside |= lo[k] > gd[3 + k] || hi[k] < gd[k];
        for (int k = 0; k < 3; k++) {
            fq[k] = grid_corner(lo[k], gd[k], gd[6], gi[1 + k]);
            lq[k] = grid_corner(hi[k], gd[k], gd[6], gi[1 + k]);
        }
    }
    const int t0 = A.mesh_tri_off[m], t1 = A.mesh_tri_off[m + 1];
    const int out0 = emit ? A.contact_scan[p] : 0;
    int count = 0;
    for (int base = t0; base < t1; base += 32) {
        const int t = base + lane;
        bool cand = false;
        if (t < t1) {
            const double *bx = &A.tri_box[(size_t)t * 6];
            if (exact) {
                cand = bx[0] <= hi[0] && bx[1] <= hi[1] && bx[2] <= hi[2] && bx[3] >= lo[0] && bx[4] >= lo[1] &&
                       bx[5] >= lo[2];
            } else if (A.tri_big[t]) {
                cand = true;
            } else if (!outside) {
                const int *tc = &A.tri_cells[(size_t)t * 6];
                cand = max(fq[0], tc[0]) <= min(lq[0], tc[3]) && max(fq[1], tc[1]) <= min(lq[1], tc[4]) &&
                       max(fq[2], tc[2]) <= min(lq[2], tc[5]);
            }
        }
        if (O.kind == 4) {
            // capsule_triangle_batch: every lane its own candidate
            bool hit = false;
            double pt[3], nr[3], dep = 0.0;
            if (cand) {
                const double *v = &A.tri_verts[(size_t)t * 9];
                const double centre[3] = {(O.e0[0] + O.e1[0]) * 0.5, (O.e0[1] + O.e1[1]) * 0.5,
                                          (O.e0[2] + O.e1[2]) * 0.5};
                hit = capsule_triangle(O.e0, O.e1, centre, O.r, v, v + 3, v + 6, pt, nr, &dep) != 0;
                if (hit && !mesh_is_a) { nr[0] = -nr[0]; nr[1] = -nr[1]; nr[2] = -nr[2]; }
            }
            const unsigned mk = __ballot_sync(FULL, hit);
            if (hit && emit) {
                const int k = out0 + count + __popc(mk & ((1u << lane) - 1u));
                if (k < A.contact_cap) {
                    A.c_a[k] = a; A.c_b[k] = b;
                    for (int c = 0; c < 3; c++) { A.c_n[k * 3 + c] = nr[c]; A.c_pt[k * 3 + c] = pt[c]; }
                    A.c_depth[k] = dep;
                    A.c_imp[k * 3] = A.c_imp[k * 3 + 1] = A.c_imp[k * 3 + 2] = 0.0;
                }
            }
            count += __popc(mk);
        } else {
            // collide_convex with a TriangleProxy, one candidate at a time,
            // the whole warp on each
            unsigned mk = __ballot_sync(FULL, cand);
            while (mk) {
                const int l = __ffs(mk) - 1;
                mk &= mk - 1;
                Proxy T;
                T.kind = 5;
                T.local = &A.tri_verts[(size_t)(base + l) * 9];
                T.m = 3;
                double nrm[3], pt[3], dep = 0.0;
                const int r = mesh_is_a ? collide_convex(T, O, W, nrm, pt, &dep, A.epa_faces)
                                         : collide_convex(O, T, W, nrm, pt, &dep, A.epa_faces);
                if (r < 0 && lane == 0 && !emit) atomicAdd(&A.status[ST_EPA_LIMIT], 1);
                if (r > 0) {
                    const int k = out0 + count;
                    if (emit && lane == 0 && k < A.contact_cap) {
                        A.c_a[k] = a; A.c_b[k] = b;
                        for (int c = 0; c < 3; c++) { A.c_n[k * 3 + c] = nrm[c]; A.c_pt[k * 3 + c] = pt[c]; }
                        A.c_depth[k] = dep;
                        A.c_imp[k * 3] = A.c_imp[k * 3 + 1] = A.c_imp[k * 3 + 2] = 0.0;
                    }
                    count++;
                }
                __syncwarp();
            }
        }
    }
    return count;
}

__global__ void k_mesh_count(Arena A) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (pairs_over(A)) return;
    EpaWork &W = reinterpret_cast<EpaWork *>(smem)[threadIdx.x >> 5];
    const int n = *A.mesh_n;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < n; it += nwarps) {
        const int p = A.mesh_list[it];
        const int cnt = mesh_pair(A, p, false, W);
        if ((threadIdx.x & 31) == 0) A.slot_cnt[p] = cnt;
        __syncwarp();
    }
}

__global__ void k_mesh_emit(Arena A) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (overflowed(A)) return;
    EpaWork &W = reinterpret_cast<EpaWork *>(smem)[threadIdx.x >> 5];
    const int n = *A.mesh_n;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < n; it += nwarps) {
        mesh_pair(A, A.mesh_list[it], true, W);
        __syncwarp();
    }
}

__global__ void k_contact_compact(Arena A) {
    if (overflowed(A)) return;
    const int P = A.pair_scan[A.NB];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const int cnt = A.slot_cnt[p];
        if (!cnt || A.pair_solid[p] == 3) continue;      // mesh pairs: k_mesh_emit
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
                                  int *last, int *level, int last_base = 0) {
    const int lane = threadIdx.x & 31;
    int maxl = -1;
    for (int base = 0; base < n; base += 32) {
        const int k = base + lane;
        const bool valid = k < n;
        const int a = valid ? ea[k] : -1, b = valid ? eb[k] : -1;
        const bool da = a >= 0 && mtype[a] == 2, db = b >= 0 && mtype[b] == 2;
        int lvl = 0;
        if (da) lvl = max(lvl, ((volatile int *)last)[a - last_base] + 1);
        if (db) lvl = max(lvl, ((volatile int *)last)[b - last_base] + 1);
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
            if (da) atomicMax(&last[a - last_base], lvl);
            if (db) atomicMax(&last[b - last_base], lvl);
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

// _effmass (_solver_native.pyx:154-176); Ia / Ib: the bodies' world inverse inertias
__device__ __forceinline__ double effmass(const double *Ia, const double *Ib, const double *ra, const double *rb,
                                          double dx, double dy, double dz, double ima, double imb) {
    const double ax = ra[1] * dz - ra[2] * dy, ay = ra[2] * dx - ra[0] * dz, az = ra[0] * dy - ra[1] * dx;
    const double bx = rb[1] * dz - rb[2] * dy, by = rb[2] * dx - rb[0] * dz, bz = rb[0] * dy - rb[1] * dx;
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
__device__ inline void prep_contact(const Arena &A, int w, int k, bool warm, int cur, double *D) {
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
    const double ima = A.inv_mass[a], imb = A.inv_mass[b];
    double Ia[9], Ib[9];
    for (int q = 0; q < 9; q++) { Ia[q] = A.invIw[a * 9 + q]; Ib[q] = A.invIw[b * 9 + q]; }
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
    D[C_RA] = rA[0]; D[C_RA + 1] = rA[1]; D[C_RA + 2] = rA[2];
    D[C_RB] = rB[0]; D[C_RB + 1] = rB[1]; D[C_RB + 2] = rB[2];
    D[R_N] = nx; D[R_N + 1] = ny; D[R_N + 2] = nz;
    D[R_T1] = t1x; D[R_T1 + 1] = t1y; D[R_T1 + 2] = t1z;
    D[R_T2] = t2x; D[R_T2 + 1] = t2y; D[R_T2 + 2] = t2z;
    D[C_NM] = effmass(Ia, Ib, rA, rB, nx, ny, nz, ima, imb);
    D[C_T1M] = effmass(Ia, Ib, rA, rB, t1x, t1y, t1z, ima, imb);
    D[C_T2M] = effmass(Ia, Ib, rA, rB, t2x, t2y, t2z, ima, imb);
    double dvx, dvy, dvz;
    rel_vel(A.v, A.w, a, b, rA, rB, dvx, dvy, dvz);
    const double vn0 = dvx * nx + dvy * ny + dvz * nz;
    D[C_VB] = vn0 < -A.w_solver[w * 2] ? -rest * vn0 : 0.0;
    D[C_DEPTH] = A.c_depth[k];
    D[11] = 0.0;
    D[R_FRIC] = fric;
    D[R_IMA] = ima;
    D[R_IMB] = imb;
    int2 *ab = reinterpret_cast<int2 *>(&D[R_AB]);
    *ab = make_int2(a, b);
    int2 *fl = reinterpret_cast<int2 *>(&D[R_FLAGS]);
    *fl = make_int2((A.mtype[a] == 2 ? 1 : 0) | (A.mtype[b] == 2 ? 2 : 0), 0);
    for (int q = 0; q < 9; q++) { D[R_IA + q] = Ia[q]; D[R_IB + q] = Ib[q]; }
}

// ---- the solver as four launches -------------------------------------------
// k_wake     one block per world, largest first: _wake_sleepers (solver.py:321-337)
// k_prep     one thread per contact, every world at once: material combine,
//            warm-start seed, arms, tangent basis, effective masses, bias
// k_levels   one block per world: runs and their predecessor / successor links
// k_iterate  persistent blocks, 1, 2 or 4 worlds each: every pass of every
//            run (warm start fused with the split-impulse position pass,
//            then the velocity iterations) as a dataflow
constexpr int WAKE_THREADS = 128;

__global__ void __launch_bounds__(WAKE_THREADS) k_wake(Arena A) {
    if (overflowed(A)) return;
    const double thr = 0.15 * 0.15;
    for (int wi = blockIdx.x; wi < A.W; wi += gridDim.x) {
        const int w = A.w_sched[wi];
        if (!world_collides(A, w) || world_wide(A, w)) continue;
        int c0, c1;
        world_contacts(A, w, c0, c1);
        if (c1 == c0) continue;
        bool cascade = false;
        for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
            const int e[2] = {A.c_a[k], A.c_b[k]};
            for (int j = 0; j < 2; j++) {
                const int x = e[j];
                cascade |= A.mtype[x] == 2 && !A.awake[x] && speed2(&A.v[x * 3]) > thr;
            }
        }
        if (__syncthreads_or(cascade)) {
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
            // no woken body can wake another (every sleeper is at rest): order
            // does not matter
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
    }
}

// one thread per contact; the block's rows (consecutive contacts) are built
// in shared memory and written out with coalesced stores
constexpr int PREP_THREADS = 128;

__global__ void __launch_bounds__(PREP_THREADS) k_prep(Arena A) {
    extern __shared__ __align__(16) double rows[];        // PREP_THREADS * CD
    __shared__ unsigned char valid[PREP_THREADS];
    if (overflowed(A)) return;
    const int cur = *A.parity;
    const int Ktot = A.contact_scan[A.pair_scan[A.NB]];
    for (int base = blockIdx.x * PREP_THREADS; base < Ktot; base += gridDim.x * PREP_THREADS) {
        const int k = base + threadIdx.x;
        bool ok = false;
        if (k < Ktot
#ifdef OMI_BOUNDS_CHECK
            && (bounds_ok(A.status, A.c_a[k], A.NB, BS_CONTACT_BODY) & bounds_ok(A.status, A.c_b[k], A.NB, BS_CONTACT_BODY))
#endif
        ) {
            const int w = A.body_world[A.c_a[k]];
            if (world_collides(A, w)) {
                prep_contact(A, w, k, (A.w_flags[w] & WF_WARM) != 0, cur, rows + threadIdx.x * CD);
                ok = true;
            }
        }
        valid[threadIdx.x] = ok;
        __syncthreads();
        const int n = min(PREP_THREADS, Ktot - base);
        double2 *dst = reinterpret_cast<double2 *>(&A.c_data[(size_t)base * CD]);
        const double2 *src = reinterpret_cast<const double2 *>(rows);
        for (int i = threadIdx.x; i < n * (CD / 2); i += PREP_THREADS)
            if (valid[i / (CD / 2)]) dst[i] = src[i];
        __syncthreads();
    }
}

// The sweep sequence. The Gauss-Seidel unit is a run (the consecutive
// contacts of one body pair) and the sequence is every pass of the
// reference's solve in order: the warm start (when on), then each velocity
// iteration, each visiting the runs in contact order. Entry (p, r) must
// follow the latest earlier entry that shares a dynamic body with it - the
// previous run of that body in the same pass, or, for the body's first run of
// the pass, its last run of pass p - 1 - and nothing else, so a run of pass
// p+1 may start while unrelated runs of pass p are still pending. The
// split-impulse position pass rides along pass 0 (it reads and writes only
// positions, which no velocity pass touches, and pass 0 orders the runs as the
// position pass does). Entries are encoded (p << 24) | r. Every run has a
// dynamic body (the broadphase keeps no pair of two static or kinematic
// bodies), so (p - 1, r) is always on a chain into (p, r).
constexpr int PASS_SHIFT = 24;
constexpr int PASS_MASK = (1 << PASS_SHIFT) - 1;

__device__ __forceinline__ int world_passes(const Arena &A, int w) {
    const int p = ((A.w_flags[w] & WF_WARM) ? 1 : 0) + A.w_iters[w];
    return p > 0 ? p : 1;
}

// ---------------------------------------------------------------------------
// Sweep dependencies of one world (one block per world).
//
// Per run and side (a dynamic body), two codes found from per-body run
// buckets: the predecessor - the previous run of that body in the same pass
// (code >= 0), or, for the body's first run of a pass, its last run of the
// previous pass (code -(run) - 1) - and the successor - the next run of that
// body in the same pass (>= 0), or, for its last run, its first run of the
// next pass (-(run) - 1). LEVEL_NONE marks a side without a dynamic body.
// The sweep itself runs the resulting graph as a dataflow.
// ---------------------------------------------------------------------------
constexpr int LEVEL_THREADS = 256;
constexpr int LEVEL_SMEM_INTS = 56 * 1024;
constexpr int LEVEL_NONE = -2147483647 - 1;

__device__ __forceinline__ void run_link_codes(const int *list, int s, int e, int r, int &pred, int &succ) {
    int pv = -1, nx = 0x7fffffff, mn = 0x7fffffff, mx = -1;
    for (int j = s; j < e; j++) {
        const int q = list[j];
        if (q < r && q > pv) pv = q;
        if (q > r && q < nx) nx = q;
        mn = min(mn, q);
        mx = max(mx, q);
    }
    pred = pv >= 0 ? pv : -(mx + 1);
    succ = nx != 0x7fffffff ? nx : -(mn + 1);
}

// block-wide exclusive scan of cnt[0..n) into out[0..n) (out may be global);
// cnt is cleared for use as a fill cursor
__device__ inline void block_scan_reset(int *cnt, int *out, int n, int *sh) {
    int carry = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < n ? cnt[i] : 0;
        int tot;
        const int x = block_exclusive_scan(v, sh, &tot);
        if (i < n) { out[i] = carry + x; cnt[i] = 0; }
        carry += tot;
    }
    __syncthreads();
}

// global scratch of world w when its buckets exceed the shared memory
__device__ __forceinline__ size_t level_scratch_offset(const Arena &A, int c0, int b0, int w) {
    return 3 * (size_t)c0 + 2 * (size_t)b0 + 2 * (size_t)w;
}

__global__ void __launch_bounds__(LEVEL_THREADS) k_levels(Arena A, int smem_ints) {
    extern __shared__ int lsm[];
    __shared__ int scan_sh[33];
    if (blockIdx.x == 0 && threadIdx.x == 0) *A.sweep_next = 0;   // the sweep's world counter
    if (overflowed(A)) return;
    const int tid = threadIdx.x, T = blockDim.x;
    for (int wi = blockIdx.x; wi < A.W; wi += gridDim.x) {
        const int w = A.w_sched[wi];
        if (!world_collides(A, w) || world_wide(A, w)) continue;
        int c0, c1;
        world_contacts(A, w, c0, c1);
        const int K = c1 - c0;
        if (K == 0 || K >= (1 << 24)) {            // run_kn packs contact offsets in 24 bits
            if (tid == 0) {
                A.w_runs[w] = 0;
                if (K) atomicOr(&A.status[ST_SWEEP_TIMEOUT], 1);
            }
            continue;
        }
        // runs: maximal stretches of consecutive contacts of one pair with one
        // normal (a solver row's pair part - normal, tangents, friction, masses
        // - is then the same for the whole run; a pair's contacts share their
        // normal except against a triangle mesh, one normal per triangle, so
        // only mesh pairs compare normals)
        int R = 0;
        for (int base = 0; base < K; base += T) {
            const int k = base + tid;
            int start = 0, a = -1, b = -1;
            if (k < K) {
                const int g = c0 + k;
                a = A.c_a[g];
                b = A.c_b[g];
                start = k == 0 || a != A.c_a[g - 1] || b != A.c_b[g - 1];
                if (!start && (A.kind[a] == 5 || A.kind[b] == 5))
                    start = A.c_n[g * 3] != A.c_n[g * 3 - 3] || A.c_n[g * 3 + 1] != A.c_n[g * 3 - 2] ||
                            A.c_n[g * 3 + 2] != A.c_n[g * 3 - 1];
            }
            int tot;
            const int r = R + block_exclusive_scan(start, scan_sh, &tot);
            if (start) {
                A.run_k[c0 + r] = k;
                A.run_a[c0 + r] = A.mtype[a] == 2 ? a : -1;
                A.run_b[c0 + r] = A.mtype[b] == 2 ? b : -1;
            }
            R += tot;
        }
        __syncthreads();
        const int b0 = A.w_body_off[w], nb = A.w_body_n[w];
        const bool in_smem = 2 * nb + 1 + 2 * R <= smem_ints;
        int *cnt = in_smem ? lsm : A.lv_scratch + level_scratch_offset(A, c0, b0, w);
        int *bstart = cnt + nb;              // nb + 1
        int *list = bstart + nb + 1;         // 2R run indices, bucketed by body
        for (int r = tid; r < R; r += T) {
            const int end = r + 1 < R ? A.run_k[c0 + r + 1] : K;
            A.run_n[c0 + r] = end - A.run_k[c0 + r];
        }
        for (int i = tid; i < nb; i += T) cnt[i] = 0;
        __syncthreads();
        for (int r = tid; r < R; r += T) {
            const int a = A.run_a[c0 + r], b = A.run_b[c0 + r];
            if (a >= 0) atomicAdd(&cnt[a - b0], 1);
            if (b >= 0) atomicAdd(&cnt[b - b0], 1);
        }
        __syncthreads();
        block_scan_reset(cnt, bstart, nb, scan_sh);
        for (int r = tid; r < R; r += T) {
            const int a = A.run_a[c0 + r], b = A.run_b[c0 + r];
            if (a >= 0) list[bstart[a - b0] + atomicAdd(&cnt[a - b0], 1)] = r;
            if (b >= 0) list[bstart[b - b0] + atomicAdd(&cnt[b - b0], 1)] = r;
        }
        __syncthreads();
        for (int r = tid; r < R; r += T) {
            const int a = A.run_a[c0 + r], b = A.run_b[c0 + r];
            int pa = LEVEL_NONE, pb = LEVEL_NONE, sa = LEVEL_NONE, sb = LEVEL_NONE;
            if (a >= 0) run_link_codes(list, bstart[a - b0], bstart[a - b0] + cnt[a - b0], r, pa, sa);
            if (b >= 0) run_link_codes(list, bstart[b - b0], bstart[b - b0] + cnt[b - b0], r, pb, sb);
            A.run_pa[c0 + r] = pa;
            A.run_pb[c0 + r] = pb;
            A.run_sa[c0 + r] = sa;
            A.run_sb[c0 + r] = sb;
            // packed for the sweep: first contact | count << 24, and the
            // same-pass / all-pass predecessor counts
            A.run_kn[c0 + r] = A.run_k[c0 + r] | (A.run_n[c0 + r] << 24);
            // (the test hook's run asks for 3 same-pass arrivals of at most 2: it never becomes ready)
            A.run_need[c0 + r] = ((pa >= 0) + (pb >= 0)) | (((pa != LEVEL_NONE) + (pb != LEVEL_NONE)) << 2) |
                                 (r == A.stall_run ? 3 : 0);
        }
        if (tid == 0) A.w_runs[w] = R;
        __syncthreads();
    }
}

// Velocities of one world, staged for the sweeps: in shared memory when the
// world fits (six doubles per body: linear then angular), else the global
// arrays. The two bodies of a pair are always distinct, so keeping their
// velocities (and, in the first pass, positions) in registers across all of
// the pair's contacts and storing them once gives exactly the arithmetic of
// updating memory after every impulse.
struct VelView {
    double *s;       // shared staging (nullptr: global)
    int b0;
};

__device__ __forceinline__ void vel_load(const Arena &A, const VelView &V, int i, double *lv, double *av) {
    if (V.s) {
        const double *p = &V.s[(i - V.b0) * 6];
        lv[0] = p[0]; lv[1] = p[1]; lv[2] = p[2]; av[0] = p[3]; av[1] = p[4]; av[2] = p[5];
    } else {
        lv[0] = A.v[i * 3]; lv[1] = A.v[i * 3 + 1]; lv[2] = A.v[i * 3 + 2];
        av[0] = A.w[i * 3]; av[1] = A.w[i * 3 + 1]; av[2] = A.w[i * 3 + 2];
    }
}
__device__ __forceinline__ void vel_store(const Arena &A, const VelView &V, int i, const double *lv,
                                          const double *av) {
    if (V.s) {
        double *p = &V.s[(i - V.b0) * 6];
        p[0] = lv[0]; p[1] = lv[1]; p[2] = lv[2]; p[3] = av[0]; p[4] = av[1]; p[5] = av[2];
    } else {
        A.v[i * 3] = lv[0]; A.v[i * 3 + 1] = lv[1]; A.v[i * 3 + 2] = lv[2];
        A.w[i * 3] = av[0]; A.w[i * 3 + 1] = av[1]; A.w[i * 3 + 2] = av[2];
    }
}

// the per-pair part of a run's row
struct PairRow {
    int a, b;
    bool da, db;
    double n[3], t1[3], t2[3], fric, ima, imb, Ia[9], Ib[9];
};
// the per-contact part
struct ContactRow {
    double rA[3], rB[3], nM, t1M, t2M, vB, depth;
};

__device__ __forceinline__ void load_pair(const double *src, PairRow &r) {
    const int2 ab = *reinterpret_cast<const int2 *>(&src[R_AB]);
    r.a = ab.x; r.b = ab.y;
    const int fl = reinterpret_cast<const int2 *>(&src[R_FLAGS])->x;
    r.da = (fl & 1) != 0; r.db = (fl & 2) != 0;
    for (int q = 0; q < 3; q++) { r.n[q] = src[R_N + q]; r.t1[q] = src[R_T1 + q]; r.t2[q] = src[R_T2 + q]; }
    r.fric = src[R_FRIC]; r.ima = src[R_IMA]; r.imb = src[R_IMB];
    for (int q = 0; q < 9; q++) { r.Ia[q] = src[R_IA + q]; r.Ib[q] = src[R_IB + q]; }
}
__device__ __forceinline__ void load_contact(const double *src, ContactRow &c) {
    for (int q = 0; q < 3; q++) { c.rA[q] = src[C_RA + q]; c.rB[q] = src[C_RB + q]; }
    c.nM = src[C_NM]; c.t1M = src[C_T1M]; c.t2M = src[C_T2M]; c.vB = src[C_VB]; c.depth = src[C_DEPTH];
}

struct PairVel {
    double la[3], aa[3], lb[3], ab[3];
};

// _apply_w (_solver_native.pyx:132-151) on the register copies
__device__ __forceinline__ void pair_apply(PairVel &s, const PairRow &r, const ContactRow &c, double Px,
                                           double Py, double Pz) {
    if (r.da) {
        s.la[0] -= r.ima * Px; s.la[1] -= r.ima * Py; s.la[2] -= r.ima * Pz;
        const double cx = c.rA[1] * Pz - c.rA[2] * Py, cy = c.rA[2] * Px - c.rA[0] * Pz, cz = c.rA[0] * Py - c.rA[1] * Px;
        s.aa[0] -= r.Ia[0] * cx + r.Ia[1] * cy + r.Ia[2] * cz;
        s.aa[1] -= r.Ia[3] * cx + r.Ia[4] * cy + r.Ia[5] * cz;
        s.aa[2] -= r.Ia[6] * cx + r.Ia[7] * cy + r.Ia[8] * cz;
    }
    if (r.db) {
        s.lb[0] += r.imb * Px; s.lb[1] += r.imb * Py; s.lb[2] += r.imb * Pz;
        const double cx = c.rB[1] * Pz - c.rB[2] * Py, cy = c.rB[2] * Px - c.rB[0] * Pz, cz = c.rB[0] * Py - c.rB[1] * Px;
        s.ab[0] += r.Ib[0] * cx + r.Ib[1] * cy + r.Ib[2] * cz;
        s.ab[1] += r.Ib[3] * cx + r.Ib[4] * cy + r.Ib[5] * cz;
        s.ab[2] += r.Ib[6] * cx + r.Ib[7] * cy + r.Ib[8] * cz;
    }
}

__device__ __forceinline__ void pair_rel_vel(const PairVel &s, const ContactRow &c, double &x, double &y, double &z) {
    x = (s.lb[0] + s.ab[1] * c.rB[2] - s.ab[2] * c.rB[1]) - (s.la[0] + s.aa[1] * c.rA[2] - s.aa[2] * c.rA[1]);
    y = (s.lb[1] + s.ab[2] * c.rB[0] - s.ab[0] * c.rB[2]) - (s.la[1] + s.aa[2] * c.rA[0] - s.aa[0] * c.rA[2]);
    z = (s.lb[2] + s.ab[0] * c.rB[1] - s.ab[1] * c.rB[0]) - (s.la[2] + s.aa[0] * c.rA[1] - s.aa[1] * c.rA[0]);
}

// warm start of one contact (_solver_native.pyx:250-256)
__device__ __forceinline__ void contact_warm(PairVel &s, const PairRow &r, const ContactRow &c, const double *imp) {
    const double n = imp[0], t0 = imp[1], t1 = imp[2];
    pair_apply(s, r, c, n * r.n[0] + t0 * r.t1[0] + t1 * r.t2[0],
               n * r.n[1] + t0 * r.t1[1] + t1 * r.t2[1],
               n * r.n[2] + t0 * r.t1[2] + t1 * r.t2[2]);
}

// one velocity-iteration update (_solver_native.pyx:259-295); imp in/out
__device__ __forceinline__ void contact_solve(PairVel &s, const PairRow &r, const ContactRow &c, double *imp) {
    double dvx, dvy, dvz;
    pair_rel_vel(s, c, dvx, dvy, dvz);
    const double vn = dvx * r.n[0] + dvy * r.n[1] + dvz * r.n[2];
    const double old = imp[0];
    double nw = old - c.nM * (vn - c.vB);
    if (nw < 0.0) nw = 0.0;
    double dL = nw - old;
    pair_apply(s, r, c, dL * r.n[0], dL * r.n[1], dL * r.n[2]);
    const double maxf = r.fric * nw;
    pair_rel_vel(s, c, dvx, dvy, dvz);
    double vt = dvx * r.t1[0] + dvy * r.t1[1] + dvz * r.t1[2];
    const double o1 = imp[1];
    double n1 = o1 - c.t1M * vt;
    if (n1 > maxf) n1 = maxf; else if (n1 < -maxf) n1 = -maxf;
    dL = n1 - o1;
    pair_apply(s, r, c, dL * r.t1[0], dL * r.t1[1], dL * r.t1[2]);
    vt = dvx * r.t2[0] + dvy * r.t2[1] + dvz * r.t2[2];
    const double o2 = imp[2];
    double n2 = o2 - c.t2M * vt;
    if (n2 > maxf) n2 = maxf; else if (n2 < -maxf) n2 = -maxf;
    dL = n2 - o2;
    pair_apply(s, r, c, dL * r.t2[0], dL * r.t2[1], dL * r.t2[2]);
    imp[0] = nw; imp[1] = n1; imp[2] = n2;
}

// split-impulse position pass of one contact (_solver_native.pyx:297-312)
__device__ __forceinline__ void contact_position(double *pa, double *pb, const PairRow &r, const ContactRow &c,
                                                 double slop) {
    const double vn = c.depth - slop;
    if (vn <= 0.0) return;
    if (r.ima + r.imb <= 1e-12) return;
    const double dL = 0.8 * vn / (r.ima + r.imb);
    if (r.da)
        for (int q = 0; q < 3; q++) pa[q] -= r.ima * dL * r.n[q];
    if (r.db)
        for (int q = 0; q < 3; q++) pb[q] += r.imb * dL * r.n[q];
}

// dynamic shared memory of one sweep block, in doubles: 227 KB less room for
// the block's static shared variables
constexpr int SWEEP_SMEM_DOUBLES = 29056 - 80;

struct ImpView {
    double *s;       // shared staging (nullptr: global c_imp)
    int c0;
};
__device__ __forceinline__ double *imp_ptr(const Arena &A, const ImpView &I, int k) {
    return I.s ? &I.s[(k - I.c0) * 3] : &A.c_imp[k * 3];
}

// the first contact's whole row (pair part included), read-only path
__device__ __forceinline__ void load_row(const Arena &A, int k, double *row) {
    const double2 *g = reinterpret_cast<const double2 *>(&A.c_data[(size_t)k * CD]);
#pragma unroll
    for (int q = 0; q < CD / 2; q++) {
        const double2 t = __ldg(g + q);
        row[2 * q] = t.x;
        row[2 * q + 1] = t.y;
    }
}

#ifdef OMI_BOUNDS_CHECK
// both bodies of a solver row inside the world's rows [b0, b0 + nb) (the
// sweep stages and indexes velocities by body - b0)
__device__ __forceinline__ bool sweep_rows_ok(const Arena &A, const double *row, int b0, int nb) {
    const int2 ab = *reinterpret_cast<const int2 *>(&row[R_AB]);
    return bounds_ok(A.status, ab.x - b0, nb, BS_SWEEP_BODY) & bounds_ok(A.status, ab.y - b0, nb, BS_SWEEP_BODY);
}
#endif

// One pass over one run (all its contacts, in order) by one thread; row0 is
// the first contact's row, the next contact's part is loaded while the
// current one is solved.
__device__ __forceinline__ void run_pass(const Arena &A, const VelView &V, const ImpView &I, const double *row0,
                                         int k0, int n, bool vel, bool warm_pass, bool pos_pass, double slop) {
    PairRow r;
    load_pair(row0, r);
    PairVel s;
    vel_load(A, V, r.a, s.la, s.aa);
    vel_load(A, V, r.b, s.lb, s.ab);
    double pa[3], pb[3];
    if (pos_pass)
        for (int q = 0; q < 3; q++) { pa[q] = A.pos[r.a * 3 + q]; pb[q] = A.pos[r.b * 3 + q]; }
    double cur[C_PART];
#pragma unroll
    for (int q = 0; q < C_PART; q++) cur[q] = row0[q];
    for (int i = 0; i < n; i++) {
        ContactRow c;
        load_contact(cur, c);
        if (i + 1 < n) {
            const double2 *g = reinterpret_cast<const double2 *>(&A.c_data[(size_t)(k0 + i + 1) * CD]);
#pragma unroll
            for (int q = 0; q < C_PART / 2; q++) {
                const double2 t = __ldg(g + q);
                cur[2 * q] = t.x;
                cur[2 * q + 1] = t.y;
            }
        }
        if (vel) {
            double *ip = imp_ptr(A, I, k0 + i);
            double imp[3] = {ip[0], ip[1], ip[2]};
            if (warm_pass) contact_warm(s, r, c, imp);
            else {
                contact_solve(s, r, c, imp);
                ip[0] = imp[0]; ip[1] = imp[1]; ip[2] = imp[2];
            }
        }
        if (pos_pass) contact_position(pa, pb, r, c, slop);
    }
    if (r.da) vel_store(A, V, r.a, s.la, s.aa);
    if (r.db) vel_store(A, V, r.b, s.lb, s.ab);
    if (pos_pass) {
        if (r.da) for (int q = 0; q < 3; q++) A.pos[r.a * 3 + q] = pa[q];
        if (r.db) for (int q = 0; q < 3; q++) A.pos[r.b * 3 + q] = pb[q];
    }
}

// block-scope acquire / release on a generic address (shared or global)
__device__ __forceinline__ int ld_acquire_cta(const int *p) {
    int v;
    asm volatile("ld.acquire.cta.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_cta(int *p, int v) {
    asm volatile("st.release.cta.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_cta() { asm volatile("fence.acq_rel.cta;" ::: "memory"); }

// Polls before a wait gives up (Arena::spin_limit, SPIN_LIMIT_DEFAULT unless
// a context lowers it): far beyond any legitimate wait (a whole world's
// sweep); one timeout sets the group's abort flag and ends every other wait
// at once.

// predecessors entry (p, r) waits for: on each side, a same-pass predecessor
// always counts, a previous-pass one only after pass 0. Runs count their
// arrivals cumulatively over the passes, so entry (p, r) is ready when
// arrivals reach need_first + p * need_rest (run_need packs both).
__device__ __forceinline__ int need_of(int pk, int p) { return (pk & 3) + p * (pk >> 2); }

// Ready entries go to one ring per class - pass 0 or not x run length 1-4 -
// so a warp claims entries that take the same path through the solve for
// the same number of contacts. Class c's ring is ring[base[c] ..) with exactly
// as many slots as the class has entries.
constexpr int SWEEP_CLASSES = 8;
// (a block shared by small worlds has few ready entries at a time: there a
// single ring keeps claims large)
__device__ __forceinline__ int entry_class(int p, int n, bool classes) {
    return classes ? (p == 0 ? 4 : 0) + min(n, 4) - 1 : 0;
}

// per-group shared scalars of the sweep
struct SweepShared {
    int head[SWEEP_CLASSES], tail[SWEEP_CLASSES], size[SWEEP_CLASSES], base[SWEEP_CLASSES];
    int claimed, abort, crit;
    bool classes;
};

// The per-world work rings: one slot per entry (each entry becomes ready
// exactly once), 0 = not yet published, else entry + 1.
__device__ __forceinline__ void sweep_push(int *ring, SweepShared &sh, int e, int n, volatile int *abort) {
    const int c = entry_class(e >> PASS_SHIFT, n, sh.classes);
    const int pos = atomicAdd(&sh.tail[c], 1);
    if (pos >= sh.size[c]) { *abort = 1; return; }    // never with a consistent graph
    st_release_cta(&ring[sh.base[c] + pos], e + 1);
}

// ---------------------------------------------------------------------------
// The sweep as a dataflow over the world's entries (SWEEP_WARPS warps per
// world). Entries whose predecessors are all done sit in the work ring; a
// warp claims up to 32 published ones at a time (CAS on the head), each lane
// solves its run, records the finish slot (for the critical-path length),
// then (after a release fence) counts itself into each successor's arrivals -
// the arrival that completes a successor fences again (acquire) and
// publishes it to the ring (release store). (Prefetching the successor's rows
// into L1 at publication cost more than it saved.) Everything an entry reads was written
// by entries that happen-before it through those release/acquire chains.
// Every wait is bounded; a timeout records ST_SWEEP_TIMEOUT and the host
// reports the step as failed. Shared memory, as far as it goes: the per-run
// arrival counts, finish slots, packed (contact, count) and need counts, the
// world's velocities, its contacts' impulses, then the work ring (else the
// global arrays).
// ---------------------------------------------------------------------------
constexpr int SWEEP_WARPS = 8;                  // default warps per sweep block (4 is the other choice)
constexpr int SWEEP_THREADS = 32 * SWEEP_WARPS;

// barrier over the `n` threads of barrier `id` (0 = the whole block)
__device__ __forceinline__ void group_sync(int id, int n) {
    if (id == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}


// shared-memory doubles one world's sweep wants: per-run tables, velocities
// and impulses (the work ring - one store and one load per entry - may
// live in global memory)
__device__ __forceinline__ int sweep_want(const Arena &A, int w) {
    int c0, c1;
    world_contacts(A, w, c0, c1);
    return 2 * A.w_runs[w] + 6 * A.w_body_n[w] + 3 * (c1 - c0) + 8;
}

// One world's sweep by the `gn` threads of a group (gtid = thread index in it,
// bar = its barrier id; 0 when the group is the whole block).
__device__ __forceinline__ void sweep_world(const Arena &A, int w, double *smem_d, int smem_doubles, int gtid, int gn, int bar,
                            SweepShared &sh) {
    const int lane = gtid & 31;
    volatile int *abort = &sh.abort;
    const int R = A.w_runs[w];
    if (R == 0) {
        if (gtid == 0) A.w_levels[w] = 0;
        return;
    }
    int c0, c1;
    world_contacts(A, w, c0, c1);
    const int K = c1 - c0;
    const int P = world_passes(A, w);
    const int N = P * R;
    const int *run_pa = A.run_pa + c0, *run_pb = A.run_pb + c0;
    const int *run_sa = A.run_sa + c0, *run_sb = A.run_sb + c0;
    const bool warm = (A.w_flags[w] & WF_WARM) != 0;
    const bool vel = warm || A.w_iters[w] > 0;
    const int b0 = A.w_body_off[w], nb = A.w_body_n[w];
    // shared memory carve-up (doubles, 16-byte multiples): per-run arrival
    // counts, finish slots, packed (contact, count) and need counts; then
    // velocities, impulses and the work ring as far as they fit
    int used = 0;
    const int runs_d = ((4 * R + 3) >> 2) << 1;
    int *arrived, *tend, *kn, *needpk;
    if (runs_d <= smem_doubles) {
        arrived = reinterpret_cast<int *>(smem_d);
        tend = arrived + R;
        kn = tend + R;
        needpk = kn + R;
        used = runs_d;
        for (int r = gtid; r < R; r += gn) {
            kn[r] = A.run_kn[c0 + r];
            needpk[r] = A.run_need[c0 + r];
        }
    } else {
        arrived = A.run_done + c0;
        tend = A.run_tend + c0;
        kn = A.run_kn + c0;
        needpk = A.run_need + c0;
    }
    VelView V;
    V.b0 = b0;
    V.s = used + nb * 6 <= smem_doubles ? smem_d + used : nullptr;
    if (V.s) used = (used + nb * 6 + 1) & ~1;
    ImpView I;
    I.c0 = c0;
    I.s = (V.s && used + K * 3 <= smem_doubles) ? smem_d + used : nullptr;
    if (I.s) used = (used + K * 3 + 1) & ~1;
    int *ring = used + ((N + 1) >> 1) <= smem_doubles ? reinterpret_cast<int *>(smem_d + used)
                                                       : A.c_order + (size_t)c0 * A.max_passes;
    if (gtid < SWEEP_CLASSES) { sh.head[gtid] = 0; sh.tail[gtid] = 0; sh.size[gtid] = 0; }
    if (gtid == 0) sh.classes = bar == 0;              // the whole block on one world
    group_sync(bar, gn);
    for (int r = gtid; r < R; r += gn) {
        arrived[r] = 0;
        tend[r] = 0;
        const int n = A.run_kn[c0 + r] >> 24;
        atomicAdd(&sh.size[entry_class(0, n, sh.classes)], 1);
        if (P > 1) atomicAdd(&sh.size[entry_class(1, n, sh.classes)], P - 1);
    }
    for (int e = gtid; e < N; e += gn) ring[e] = 0;
    if (V.s) {
        for (int i = gtid; i < nb; i += gn) {
            double lv[3], av[3];
            lv[0] = A.v[(b0 + i) * 3]; lv[1] = A.v[(b0 + i) * 3 + 1]; lv[2] = A.v[(b0 + i) * 3 + 2];
            av[0] = A.w[(b0 + i) * 3]; av[1] = A.w[(b0 + i) * 3 + 1]; av[2] = A.w[(b0 + i) * 3 + 2];
            vel_store(A, V, b0 + i, lv, av);
        }
    }
    if (I.s)
        for (int i = gtid; i < K * 3; i += gn) I.s[i] = A.c_imp[c0 * 3 + i];
    group_sync(bar, gn);
    if (gtid == 0) {
        int acc = 0;
        for (int c = 0; c < SWEEP_CLASSES; c++) { sh.base[c] = acc; acc += sh.size[c]; }
        sh.claimed = 0; sh.abort = 0; sh.crit = 0;
    }
    group_sync(bar, gn);
    // entries with no predecessor: pass-0 runs that start both bodies' chains
    for (int r = gtid; r < R; r += gn)
        if ((needpk[r] & 3) == 0) sweep_push(ring, sh, r, kn[r] >> 24, abort);
    group_sync(bar, gn);
    const double slop = A.w_solver[w * 2 + 1];
    int my_crit = 0;
    for (;;) {
        // lane 0 claims up to 32 published-or-pending positions of one class
        int lo = 0, cnt = 0;
        if (lane == 0) {
            const int first = (gtid >> 5) & (SWEEP_CLASSES - 1);
            for (int it = 0;; it++) {
                if (*(volatile int *)&sh.claimed >= N || *abort) { cnt = -1; break; }
                bool got = false;
                for (int j = 0; j < SWEEP_CLASSES && !got; j++) {
                    const int c = (first + j) & (SWEEP_CLASSES - 1);
                    const int h = *(volatile int *)&sh.head[c];
                    const int t = min(*(volatile int *)&sh.tail[c], sh.size[c]);
                    if (t > h) {
                        const int want = min(t - h, A.sweep_claim);
                        if (atomicCAS(&sh.head[c], h, h + want) == h) {
                            atomicAdd(&sh.claimed, want);
                            lo = sh.base[c] + h;
                            cnt = want;
                            got = true;
                        }
                    }
                }
                if (got) break;
                if (it >= A.spin_limit) { *abort = 1; cnt = -1; break; }
                __nanosleep(32);
            }
        }
        cnt = __shfl_sync(FULL, cnt, 0);
        lo = __shfl_sync(FULL, lo, 0);
        if (cnt < 0) break;
        if (lane < cnt) {
            int e1 = 0;
            for (int it = 0; it < A.spin_limit; it++) {   // the pusher is between its two steps
                e1 = ld_acquire_cta(&ring[lo + lane]);
                if (e1 || *abort) break;
            }
            if (e1 == 0) *abort = 1;
            else {
                const int e = e1 - 1;
                const int r = e & PASS_MASK, p = e >> PASS_SHIFT;
                const int v = kn[r];
                const int k0 = c0 + (v & 0xFFFFFF), n = v >> 24;
                double row0[CD];
                load_row(A, k0, row0);
                // codes for the finish slot and the successors, loaded during the solve
                const int ca = __ldg(run_pa + r), cb = __ldg(run_pb + r);
                const int sa = __ldg(run_sa + r), sb = __ldg(run_sb + r);
#ifdef OMI_BOUNDS_CHECK
                if (sweep_rows_ok(A, row0, b0, nb))
#endif
                run_pass(A, V, I, row0, k0, n, vel, warm && p == 0, p == 0, slop);
                // finish slot (critical-path diagnostics), off the solve's path
                int t0 = 0;
                if (ca >= 0) t0 = tend[ca]; else if (ca != LEVEL_NONE && p > 0) t0 = tend[-ca - 1];
                if (cb >= 0) t0 = max(t0, tend[cb]); else if (cb != LEVEL_NONE && p > 0) t0 = max(t0, tend[-cb - 1]);
                tend[r] = t0 + n;
                my_crit = max(my_crit, t0 + n);
                // release this entry's writes, then count into the successors
                fence_acq_rel_cta();
                const int sides[2] = {sa, sb};
#pragma unroll
                for (int sd = 0; sd < 2; sd++) {
                    const int sc = sides[sd];
                    int ps, rs;
                    if (sc >= 0) { ps = p; rs = sc; }
                    else if (sc != LEVEL_NONE && p + 1 < P) { ps = p + 1; rs = -sc - 1; }
                    else continue;
                    OMI_BOUNDS(A, rs, R, BS_SWEEP_RUN, continue)
                    if (atomicAdd(&arrived[rs], 1) + 1 == need_of(needpk[rs], ps)) {
                        fence_acq_rel_cta();             // acquire the other arrivals' writes
                        sweep_push(ring, sh, (ps << PASS_SHIFT) | rs, kn[rs] >> 24, abort);
                    }
                }
            }
        }
        __syncwarp();
    }
    atomicMax(&sh.crit, my_crit);
    group_sync(bar, gn);
    if (gtid == 0) {
        A.w_levels[w] = sh.crit;
        if (sh.abort || sh.claimed < N) atomicOr(&A.status[ST_SWEEP_TIMEOUT], 1);
    }
    if (V.s) {
        for (int i = gtid; i < nb; i += gn) {
            if (A.mtype[b0 + i] != 2) continue;
            double lv[3], av[3];
            vel_load(A, V, b0 + i, lv, av);
            A.v[(b0 + i) * 3] = lv[0]; A.v[(b0 + i) * 3 + 1] = lv[1]; A.v[(b0 + i) * 3 + 2] = lv[2];
            A.w[(b0 + i) * 3] = av[0]; A.w[(b0 + i) * 3 + 1] = av[1]; A.w[(b0 + i) * 3 + 2] = av[2];
        }
    }
    if (I.s)
        for (int i = gtid; i < K * 3; i += gn) A.c_imp[c0 * 3 + i] = I.s[i];
    group_sync(bar, gn);
}

// Persistent sweep blocks take worlds in schedule order (largest first) from
// a counter k_levels reset. While the worlds taken need the whole block's
// shared memory, the block sweeps them one at a time. The first world whose
// needs fit a half (or a quarter) splits the block into 2 (or 4) groups for
// good: every later world is no larger, so from then on each group takes its
// own next world as soon as it is done, with no block-wide barrier between
// worlds.
constexpr int SWEEP_MAX_GROUPS = 4;

// next colliding world of the schedule, or -1
__device__ __forceinline__ int sweep_take(const Arena &A) {
    for (;;) {
        const int wi = atomicAdd(A.sweep_next, 1);
        if (wi >= A.W) return -1;
        const int w = A.w_sched[wi];
        if (world_collides(A, w) && !world_wide(A, w)) return w;
    }
}

// WARPS warps per block (a launch-configuration choice); max_split caps the
// groups a block splits into (1, 2 or 4)
template <int WARPS>
__global__ void __launch_bounds__(32 * WARPS) k_iterate(Arena A, int smem_doubles, int max_split) {
    extern __shared__ __align__(16) double smem_d[];
    __shared__ SweepShared sh[SWEEP_MAX_GROUPS];
    __shared__ int pick[1 + SWEEP_MAX_GROUPS];    // split (0: done), world per group
    if (overflowed(A)) return;
    constexpr int THREADS = 32 * WARPS;
    const int tid = threadIdx.x;
    int G;
    for (;;) {
        if (tid == 0) {
            const int w = sweep_take(A);
            int g = 0;
            if (w >= 0) {
                const int want = sweep_want(A, w);
                g = (max_split >= 4 && want <= ((smem_doubles / 4) & ~1)) ? 4
                    : ((max_split >= 2 && want <= ((smem_doubles / 2) & ~1)) ? 2 : 1);
                g = min(g, WARPS);                  // at least one warp per group
            }
            pick[0] = g;
            pick[1] = w;
        }
        __syncthreads();
        G = pick[0];
        if (G == 0) return;
        if (G > 1) break;
        sweep_world(A, pick[1], smem_d, smem_doubles, tid, THREADS, 0, sh[0]);
        __syncthreads();
    }
    // split for good: group g sweeps its own worlds on named barrier 1 + g
    const int gn = THREADS / G, g = tid / gn, gtid = tid - g * gn;
    const int share = (smem_doubles / G) & ~1;
    int w = g == 0 ? pick[1] : -1;
    for (;;) {
        if (w < 0) {
            group_sync(1 + g, gn);                 // everyone has read the previous pick
            if (gtid == 0) pick[1 + g] = sweep_take(A);
            group_sync(1 + g, gn);
            w = pick[1 + g];
            if (w < 0) return;
        }
        sweep_world(A, w, smem_d + g * share, share, gtid, gn, 1 + g, sh[g]);
        w = -1;
    }
}

}  // namespace omi
