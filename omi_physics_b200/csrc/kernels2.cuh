// Warm-start cache store, joints, and the integrate-positions + sleep pass.
#pragma once
#include "kernels.cuh"

namespace omi {

// ---------------------------------------------------------------------------
// warm-start cache (solver.py:91, 271-278). A world that had contacts this
// step (and warm starting on) replaces its cache with them; any other world
// keeps its previous cache, as the reference does when solve() returns early.
// The cache is double-buffered; a hash table per buffer maps a body pair to
// its run of entries.
// ---------------------------------------------------------------------------
__global__ void k_cache_plan(Arena A) {   // one CTA
    __shared__ int sh[32];
    if (overflowed(A)) return;
    const int cur = *A.parity, nxt = 1 - cur;
    int carry = 0;
    for (int base = 0; base < A.W; base += blockDim.x) {
        const int w = base + threadIdx.x;
        int n_new = 0;
        if (w < A.W) {
            int K = 0;
            if (world_collides(A, w)) {
                int c0, c1;
                world_contacts(A, w, c0, c1);
                K = c1 - c0;
            }
            const bool refresh = K > 0 && (A.w_flags[w] & WF_WARM) && world_collides(A, w);
            n_new = refresh ? K : A.w_cache_n[cur][w];
            A.w_cache_new[w] = refresh ? 1 : 0;
        }
        int total;
        const int pre = block_exclusive_scan(n_new, sh, &total) + carry;
        if (w < A.W) { A.w_cache_off[nxt][w] = pre; A.w_cache_n[nxt][w] = n_new; }
        carry += total;
    }
    if (threadIdx.x == 0) {
        A.hused_n[2] = A.hused_n[nxt];   // slots of table nxt to clear
        A.hused_n[nxt] = 0;
    }
}

__global__ void k_hash_clear(Arena A) {
    if (overflowed(A)) return;
    const int nxt = 1 - *A.parity;
    const int n = A.hused_n[2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        A.hkey[nxt][A.hused[nxt][i]] = ~0ull;
}

// entry e of world w in the next cache buffer: this step's contact c0 + e
// when the world refreshes its cache, else the entry kept from the current one
__device__ __forceinline__ void cache_copy_entry(const Arena &A, int w, int cur, int e) {
    const int nxt = 1 - cur;
    const int d = A.w_cache_off[nxt][w] + e;
    if (A.w_cache_new[w]) {
        int c0, c1;
        world_contacts(A, w, c0, c1);
        const int k = c0 + e;
        A.cache_a[nxt][d] = A.c_a[k];
        A.cache_b[nxt][d] = A.c_b[k];
        for (int c = 0; c < 3; c++) {
            A.cache_pt[nxt][d * 3 + c] = A.c_pt[k * 3 + c];
            A.cache_imp[nxt][d * 3 + c] = A.c_imp[k * 3 + c];
        }
    } else {
        const int s = A.w_cache_off[cur][w] + e;
        A.cache_a[nxt][d] = A.cache_a[cur][s];
        A.cache_b[nxt][d] = A.cache_b[cur][s];
        for (int c = 0; c < 3; c++) {
            A.cache_pt[nxt][d * 3 + c] = A.cache_pt[cur][s * 3 + c];
            A.cache_imp[nxt][d * 3 + c] = A.cache_imp[cur][s * 3 + c];
        }
    }
}

// entries of buffer t in use: the worlds' entries are packed in world order
__device__ __forceinline__ int cache_total(const Arena &A, int t) {
    return A.W > 0 ? A.w_cache_off[t][A.W - 1] + A.w_cache_n[t][A.W - 1] : 0;
}

// the world that entry d of buffer t belongs to: the last world whose first
// entry is at or before d (an empty world shares its offset with the next
// world, which is the one that holds d)
__device__ __forceinline__ int cache_world(const Arena &A, int t, int d) {
    int lo = 0, hi = A.W;
    while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (A.w_cache_off[t][m] <= d) lo = m + 1; else hi = m;
    }
    return lo - 1;
}

// Every world's entries of the next buffer, one thread per entry over the
// whole grid (a world's entries no longer wait for one CTA to stride through
// them; the largest world set the time of the CTA-per-world form).
__global__ void k_cache_copy(Arena A) {
    if (overflowed(A)) return;
    const int cur = *A.parity, nxt = 1 - cur;
    const int total = cache_total(A, nxt);
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < total; d += gridDim.x * blockDim.x) {
        const int w = cache_world(A, nxt, d);
        cache_copy_entry(A, w, cur, d - A.w_cache_off[nxt][w]);
    }
}

// insert one key per run of equal (a, b) entries of buffer t's range
// [lo, hi) into table t, looking at entries lo + first, lo + first + stride, ...
__device__ inline void hash_range(const Arena &A, int t, int lo, int hi, int first, int stride) {
    const int *ca = A.cache_a[t], *cb = A.cache_b[t];
    for (int e = lo + first; e < hi; e += stride) {
        if (e > lo && ca[e] == ca[e - 1] && cb[e] == cb[e - 1]) continue;
        int len = 1;
        while (e + len < hi && ca[e + len] == ca[e] && cb[e + len] == cb[e]) len++;
        const unsigned long long key = pair_key(ca[e], cb[e]);
        int s = hash_slot(key, A.hash_mask), fresh = -1;
        for (int probe = 0; probe <= A.hash_mask; probe++) {
            const unsigned long long prev = atomicCAS(&A.hkey[t][s], ~0ull, key);
            if (prev == ~0ull || prev == key) {
                A.hval[t][s * 2] = e;
                A.hval[t][s * 2 + 1] = len;
                if (prev == ~0ull) fresh = s;
                break;
            }
            s = (s + 1) & A.hash_mask;
        }
        if (fresh >= 0) A.hused[t][list_slot(&A.hused_n[t])] = fresh;   // the slots the next clear empties
    }
}

// world w's runs (a CTA per world)
__device__ inline void hash_runs(const Arena &A, int t, int w, int first, int stride) {
    const int off = A.w_cache_off[t][w];
    hash_range(A, t, off, off + A.w_cache_n[t][w], first, stride);
}

// Every world's runs at once, over the whole grid, table = next buffer. Body
// indices are global and no two worlds share a body, so a run (one body
// pair) never reaches into the next world: scanning the packed buffer as
// one range finds exactly the runs the per-world scan finds.
__global__ void k_hash_build(Arena A) {
    if (overflowed(A)) return;
    const int nxt = 1 - *A.parity;
    hash_range(A, nxt, 0, cache_total(A, nxt), blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__global__ void k_flip(Arena A) {
    if (overflowed(A)) return;
    *A.parity = 1 - *A.parity;
}

// rebuild table t from cache buffer t (after the host regrows the tables)
__global__ void k_hash_rebuild(Arena A, int t) {
    for (int w = blockIdx.x; w < A.W; w += gridDim.x) hash_runs(A, t, w, threadIdx.x, blockDim.x);
}

// ---------------------------------------------------------------------------
// joints (world.py:599-611, joints.py:60-212), one warp per world; prepare in
// parallel, then every joint iteration in registration order, as wavefront
// levels
// ---------------------------------------------------------------------------
enum { J_IA = 0, J_IB = 9, J_RA = 18, J_RB = 21, J_LU = 24, J_PIV = 33, J_BIAS = 36, J_N = 39,
       J_MASS = 42, J_BIASS = 43 };
// joint iterations the wavefront schedule buffers hold per joint (a world
// with more iterations sweeps iteration by iteration)
constexpr int JOINT_WAVE_ITERS = 32;

// joints.py:278-283: (R * invI) @ R.T through BLAS; zero for the world (-1)
__device__ inline void joint_inv_inertia(const Arena &A, int i, double *W) {
    if (i < 0) { for (int q = 0; q < 9; q++) W[q] = 0.0; return; }
    double R[9], s[9];
    quat_to_matrix(&A.q[i * 4], R);
    const double *ii = &A.inv_inertia[i * 3];
    for (int r = 0; r < 3; r++)
        for (int j = 0; j < 3; j++) s[r * 3 + j] = R[r * 3 + j] * ii[j];
    for (int r = 0; r < 3; r++)
        for (int k = 0; k < 3; k++) W[r * 3 + k] = dot_blas(&s[r * 3], &R[k * 3]);
}

__device__ inline void mat3_mul(const double *X, const double *Y, double *Z) {
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            const double col[3] = {Y[k], Y[3 + k], Y[6 + k]};
            Z[i * 3 + k] = dot_blas(&X[i * 3], col);
        }
}

__device__ inline void skew(const double *r, double *S) {
    S[0] = 0.0; S[1] = -r[2]; S[2] = r[1];
    S[3] = r[2]; S[4] = 0.0; S[5] = -r[0];
    S[6] = -r[1]; S[7] = r[0]; S[8] = 0.0;
}

// prepares joint j's row into D (JD doubles: shared memory or j_data)
__device__ inline void joint_prepare(const Arena &A, int j, double *D) {
    const int t = A.j_type[j];
    if (t == 2) {                                    // AngularMotor.prepare
        const int body = A.j_a[j];
        joint_inv_inertia(A, body, &D[J_IA]);
        const double *ax = &A.j_axis[j * 3];
        double u[3];
        for (int k = 0; k < 3; k++) {
            const double col[3] = {D[J_IA + k], D[J_IA + 3 + k], D[J_IA + 6 + k]};
            u[k] = dot_blas(ax, col);
        }
        const double eff = dot_blas(u, ax);
        D[J_MASS] = eff > 1e-12 ? 1.0 / eff : 0.0;
        A.j_accum[j] = 0.0;
        return;
    }
    const int a = A.j_a[j], b = A.j_b[j];
    joint_inv_inertia(A, a, &D[J_IA]);
    joint_inv_inertia(A, b, &D[J_IB]);
    if (t == 0) {                                    // PointConstraint.prepare
        const double *anchor = &A.j_anchor[j * 3];
        const int ids[2] = {a, b};
        double *locs[2] = {&A.j_local_a[j * 3], &A.j_local_b[j * 3]};
        uint8_t *has[2] = {&A.j_has_local_a[j], &A.j_has_local_b[j]};
        double posv[2][3];
        for (int e = 0; e < 2; e++) {
            const int i = ids[e];
            double *r = &D[e == 0 ? J_RA : J_RB];
            if (i < 0) {
                for (int k = 0; k < 3; k++) { posv[e][k] = anchor[k]; r[k] = anchor[k] - anchor[k]; }
                continue;
            }
            double R[9];
            quat_to_matrix(&A.q[i * 4], R);
            if (!*has[e]) {                          // _to_local: R.T @ (anchor - pos)
                double dd[3];
                sub3(anchor, &A.pos[i * 3], dd);
                for (int k = 0; k < 3; k++) {
                    const double col[3] = {R[k], R[3 + k], R[6 + k]};
                    locs[e][k] = dot_blas(col, dd);
                }
                *has[e] = 1;
            }
            for (int k = 0; k < 3; k++) {
                posv[e][k] = A.pos[i * 3 + k];
                r[k] = (A.pos[i * 3 + k] + gemv_row(&R[k * 3], locs[e])) - posv[e][k];
            }
        }
        const double im = (a < 0 ? 0.0 : A.inv_mass[a]) + (b < 0 ? 0.0 : A.inv_mass[b]);
        double K[9], S[9], T[9], M[9];
        for (int q = 0; q < 9; q++) K[q] = (q % 4 == 0) ? im * 1.0 : im * 0.0;
        skew(&D[J_RA], S); mat3_mul(S, &D[J_IA], T); mat3_mul(T, S, M);
        for (int q = 0; q < 9; q++) K[q] = K[q] - M[q];
        skew(&D[J_RB], S); mat3_mul(S, &D[J_IB], T); mat3_mul(T, S, M);
        for (int q = 0; q < 9; q++) K[q] = K[q] - M[q];
        for (int k = 0; k < 3; k++) {
            const double pa = posv[0][k] + D[J_RA + k], pb = posv[1][k] + D[J_RB + k];
            D[J_BIAS + k] = 0.2 * (pb - pa);
        }
        // LU with partial pivoting of K, kept for every iteration's solve
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
            int p = jj;
            double best = fabs(K[jj * 3 + jj]);
#pragma unroll
            for (int i = jj + 1; i < 3; i++)
                if (fabs(K[i * 3 + jj]) > best) { best = fabs(K[i * 3 + jj]); p = i; }
            D[J_PIV + jj] = (double)p;
            // row swap with static indices (a dynamic one would put K in local memory)
#pragma unroll
            for (int i = jj + 1; i < 3; i++)
                if (p == i)
#pragma unroll
                    for (int k = 0; k < 3; k++) { const double tt = K[jj * 3 + k]; K[jj * 3 + k] = K[i * 3 + k]; K[i * 3 + k] = tt; }
#pragma unroll
            for (int i = jj + 1; i < 3; i++) {
                const double l = K[i * 3 + jj] / K[jj * 3 + jj];
                K[i * 3 + jj] = l;
                for (int k = jj + 1; k < 3; k++) K[i * 3 + k] = fma(-l, K[jj * 3 + k], K[i * 3 + k]);
            }
        }
        for (int q = 0; q < 9; q++) D[J_LU + q] = K[q];
        return;
    }
    // DistanceConstraint.prepare
    const double *la = &A.j_anchor[j * 3], *lb = &A.j_anchor_b[j * 3];
    double pa[3], pb[3], d[3];
    for (int e = 0; e < 2; e++) {
        const int i = e == 0 ? a : b;
        const double *loc = e == 0 ? la : lb;
        double *out = e == 0 ? pa : pb;
        if (i < 0) { for (int k = 0; k < 3; k++) out[k] = loc[k]; }
        else {
            double R[9];
            quat_to_matrix(&A.q[i * 4], R);
            for (int k = 0; k < 3; k++) out[k] = A.pos[i * 3 + k] + gemv_row(&R[k * 3], loc);
        }
    }
    sub3(pb, pa, d);
    const double dist = sqrt(dot_blas(d, d));
    double *n = &D[J_N];
    if (dist > 1e-9) { for (int k = 0; k < 3; k++) n[k] = d[k] / dist; }
    else { n[0] = 0.0; n[1] = 1.0; n[2] = 0.0; }
    if (!A.j_has_length[j]) { A.j_length[j] = dist; A.j_has_length[j] = 1; }
    for (int k = 0; k < 3; k++) {
        D[J_RA + k] = pa[k] - (a < 0 ? la[k] : A.pos[a * 3 + k]);
        D[J_RB + k] = pb[k] - (b < 0 ? la[k] : A.pos[b * 3 + k]);
    }
    double raxn[3], rbxn[3], u[3];
    cross_np(&D[J_RA], n, raxn);
    cross_np(&D[J_RB], n, rbxn);
    double k = (a < 0 ? 0.0 : A.inv_mass[a]) + (b < 0 ? 0.0 : A.inv_mass[b]);
    for (int q = 0; q < 3; q++) { const double col[3] = {D[J_IA + q], D[J_IA + 3 + q], D[J_IA + 6 + q]}; u[q] = dot_blas(raxn, col); }
    k += dot_blas(u, raxn);
    for (int q = 0; q < 3; q++) { const double col[3] = {D[J_IB + q], D[J_IB + 3 + q], D[J_IB + 6 + q]}; u[q] = dot_blas(rbxn, col); }
    k += dot_blas(u, rbxn);
    D[J_MASS] = k > 1e-12 ? 1.0 / k : 0.0;
    D[J_BIASS] = 0.2 * (dist - A.j_length[j]);
}

// where the joint solve reads and writes body velocities: a world's range
// [lo, lo + n) of bodies staged in shared memory (v then w, 6 per body), or
// the global arrays (s == nullptr)
struct JointVel {
    double *s;
    int lo;
    __device__ __forceinline__ double *v(const Arena &A, int i) const { return s ? s + (i - lo) * 6 : &A.v[i * 3]; }
    __device__ __forceinline__ double *w(const Arena &A, int i) const { return s ? s + (i - lo) * 6 + 3 : &A.w[i * 3]; }
};

__device__ inline void joint_apply(const Arena &A, const JointVel &V, int i, const double *invI, const double *r,
                                   const double *P) {
    if (i < 0 || A.mtype[i] != 2) return;
    double *v = V.v(A, i), *w = V.w(A, i);
    for (int q = 0; q < 3; q++) v[q] = v[q] + A.inv_mass[i] * P[q];
    double c[3];
    cross_np(r, P, c);
    for (int q = 0; q < 3; q++) w[q] = w[q] + gemv_row(&invI[q * 3], c);
}

// one solve of joint j (prepared row D) on the velocities V
__device__ inline void joint_solve(const Arena &A, int j, const double *D, const JointVel &V, double dt) {
    const int t = A.j_type[j];
    if (t == 2) {                                    // AngularMotor.solve
        const int body = A.j_a[j];
        if (body < 0) return;
        const double *ax = &A.j_axis[j * 3];
        double *wb = V.w(A, body);
        const double wv = dot_blas(wb, ax);
        double impulse = D[J_MASS] * (A.j_target[j] - wv);
        const double limit = A.j_max_force[j] * dt;
        double nw = A.j_accum[j] + impulse;
        if (nw < -limit) nw = -limit;
        if (nw > limit) nw = limit;
        impulse = nw - A.j_accum[j];
        A.j_accum[j] = nw;
        if (A.mtype[body] != 2) return;
        const double P[3] = {ax[0] * impulse, ax[1] * impulse, ax[2] * impulse};
        for (int q = 0; q < 3; q++) wb[q] = wb[q] + gemv_row(&D[J_IA + q * 3], P);
        return;
    }
    const int a = A.j_a[j], b = A.j_b[j];
    double va[3] = {0.0, 0.0, 0.0}, vb[3] = {0.0, 0.0, 0.0}, P[3], nP[3], c[3];
    if (b >= 0) { cross_np(V.w(A, b), &D[J_RB], c); const double *v = V.v(A, b); for (int q = 0; q < 3; q++) vb[q] = v[q] + c[q]; }
    if (a >= 0) { cross_np(V.w(A, a), &D[J_RA], c); const double *v = V.v(A, a); for (int q = 0; q < 3; q++) va[q] = v[q] + c[q]; }
    if (t == 0) {                                    // PointConstraint.solve
        double x[3];
        for (int q = 0; q < 3; q++) x[q] = -((vb[q] - va[q]) + D[J_BIAS + q] / dt);
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
            const int p = (int)D[J_PIV + jj];
#pragma unroll
            for (int i = jj + 1; i < 3; i++)           // static indices: x stays in registers
                if (p == i) { const double tt = x[jj]; x[jj] = x[i]; x[i] = tt; }
        }
        const double *L = &D[J_LU];
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < i; k++) x[i] = fma(-L[i * 3 + k], x[k], x[i]);
        for (int i = 2; i >= 0; i--) {
            for (int k = i + 1; k < 3; k++) x[i] = fma(-L[i * 3 + k], x[k], x[i]);
            x[i] = x[i] / L[i * 3 + i];
        }
        P[0] = x[0]; P[1] = x[1]; P[2] = x[2];
    } else {                                         // DistanceConstraint.solve
        double dv[3];
        sub3(vb, va, dv);
        const double cdot = dot_blas(dv, &D[J_N]);
        const double impulse = -D[J_MASS] * (cdot + D[J_BIASS] / dt);
        for (int q = 0; q < 3; q++) P[q] = impulse * D[J_N + q];
    }
    neg3(P, nP);
    joint_apply(A, V, a, &D[J_IA], &D[J_RA], nP);
    joint_apply(A, V, b, &D[J_IB], &D[J_RB], P);
}

// A motor whose body is not dynamic changes only its own accumulated impulse
// (it reads that body's constant angular velocity and writes nothing else).
__device__ __forceinline__ bool motor_alone(const Arena &A, int j) {
    return A.j_type[j] == 2 && (A.j_a[j] < 0 || A.mtype[A.j_a[j]] != 2);
}

// Wavefront levels of all joint iterations of one world (one warp): entry
// e = it * J + jj is joint jj in iteration it; its level is one more than
// that of the latest earlier entry, in the reference's order (iteration by
// iteration, joints in registration order), sharing a dynamic body with it.
// Iteration it + 1 of a joint so starts as soon as its own bodies are done
// with iteration it: a chain of J joints takes about J + 2 * iters levels
// instead of iters * J. A lone motor (motor_alone) runs all its iterations in
// its iteration-0 entry, at level 0. Entries of one level share no dynamic
// body, so running the levels in order repeats the sequential arithmetic.
__device__ inline int warp_joint_levels(const Arena &A, int j0, int J, int iters, int *last, int *level,
                                        int last_base) {
    const int lane = threadIdx.x & 31;
    const int n = J * iters;
    int maxl = -1;
    for (int base = 0; base < n; base += 32) {
        const int e = base + lane;
        const bool valid = e < n;
        int a = -1, b = -1;
        if (valid) {
            const int j = j0 + e % J;
            a = A.j_a[j];
            b = A.j_type[j] == 2 ? -1 : A.j_b[j];
        }
        const bool da = a >= 0 && A.mtype[a] == 2, db = b >= 0 && A.mtype[b] == 2;
        int lvl = 0;
        if (da) lvl = max(lvl, ((volatile int *)last)[a - last_base] + 1);
        if (db) lvl = max(lvl, ((volatile int *)last)[b - last_base] + 1);
        unsigned conflict = 0;
        for (int q = 0; q < 32; q++) {
            const int aq = __shfl_sync(FULL, a, q), bq = __shfl_sync(FULL, b, q);
            const bool c = q < lane && ((da && (a == aq || a == bq)) || (db && (b == aq || b == bq)));
            conflict |= (c ? 1u : 0u) << q;
        }
        for (int q = 0; q < 32; q++) {
            const int lq = __shfl_sync(FULL, lvl, q);
            if ((conflict >> q) & 1u) lvl = max(lvl, lq + 1);
        }
        if (valid) {
            level[e] = lvl;
            if (da) atomicMax(&last[a - last_base], lvl);
            if (db) atomicMax(&last[b - last_base], lvl);
            maxl = max(maxl, lvl);
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) maxl = max(maxl, __shfl_xor_sync(FULL, maxl, o));
    return maxl + 1;
}

// shared memory of one k_joints block (one world at a time), in doubles, at
// most: the launch sizes it to the scene's largest need (joint_smem_need);
// a 128-link chain at 12 iterations needs about 8.7K (rows 6.1K, velocities
// 0.8K, schedule 1.8K), so three blocks fit on an SM
constexpr int JOINT_SMEM_DOUBLES = 13312;

// inclusive prefix sums of a[0..n) by one warp (each lane sums a chunk)
__device__ inline void warp_scan_inclusive(int *a, int n) {
    const int lane = threadIdx.x & 31;
    const int per = (n + 31) >> 5;
    const int s0 = min(lane * per, n), s1 = min(s0 + per, n);
    int sum = 0;
    for (int i = s0; i < s1; i++) sum += a[i];
    int x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    int run = x - sum;
    for (int i = s0; i < s1; i++) {
        run += a[i];
        a[i] = run;
    }
    __syncwarp();
}

// _solve_joints (world.py:599-611): wake, prepare, then every joint
// iteration in the reference's order, as wavefront levels. One warp per world
// (one block of 32 threads): a chain's levels hold a few entries each (about
// one per iteration in flight), so a warp fills them and steps from level to
// level with __syncwarp alone. The prepared rows, the joints' body
// velocities and the schedule (levels, order, level starts) live in the
// block's shared memory as far as `smem_doubles` goes, else in the global
// arrays (rows in L1 lose to shared memory: the solve stalls on them); the
// velocities go back to the global arrays at the end.
__global__ void __launch_bounds__(32, 1) k_joints(Arena A, int gated, int smem_doubles) {
    extern __shared__ __align__(16) double jsm[];
    if (gated && overflowed(A)) return;
    const int lane = threadIdx.x & 31;
    for (int w = blockIdx.x; w < A.W; w += gridDim.x) {
        if (!A.w_active[w]) continue;
        const int j0 = A.w_joint_off[w], J = A.w_joint_n[w], j1 = j0 + J;
        if (J == 0) continue;
#ifdef OMI_BOUNDS_CHECK
        {   // every joint body inside the world's rows, else the world's joints are skipped
            const int b0 = A.w_body_off[w], nb = A.w_body_n[w];
            bool bad = false;
            for (int j = j0 + lane; j < j1; j += 32) {
                if (A.j_a[j] >= 0 && !bounds_ok(A.status, A.j_a[j] - b0, nb, BS_JOINT_BODY)) bad = true;
                if (A.j_b[j] >= 0 && !bounds_ok(A.status, A.j_b[j] - b0, nb, BS_JOINT_BODY)) bad = true;
            }
            if (__any_sync(FULL, bad)) continue;
        }
#endif
        const double dt = A.w_dt[w];
        const int iters = A.w_jiters[w];
        const bool waves = iters <= JOINT_WAVE_ITERS;   // the schedule buffers hold that many iterations
        const int E = waves ? J * iters : J;
        // the joints' bodies span [lo, hi]
        int lo = 0x7FFFFFFF, hi = -1;
        for (int j = j0 + lane; j < j1; j += 32) {
            const int a = A.j_a[j], b = A.j_b[j];
            if (a >= 0) { lo = min(lo, a); hi = max(hi, a); }
            if (b >= 0) { lo = min(lo, b); hi = max(hi, b); }
        }
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(FULL, lo, o));
            hi = max(hi, __shfl_xor_sync(FULL, hi, o));
        }
        const int nbr = hi >= lo ? hi - lo + 1 : 0;
        // shared memory: the prepared rows, the velocities, the levels and the
        // order, then (once the level count is known) the level starts; each
        // in the global arrays when it does not fit
        long long used = 0;
        double *rows = nullptr;
        if ((long long)J * JD <= smem_doubles) { rows = jsm; used = (long long)J * JD; }
        JointVel V;
        V.s = nullptr;
        V.lo = lo;
        if (nbr > 0 && used + 6LL * nbr <= smem_doubles) { V.s = jsm + used; used += 6LL * nbr; }
        int *ip = reinterpret_cast<int *>(jsm + used);
        const long long ints_free = 2LL * (smem_doubles - used);
        int *last, *lvl, *order;
        int last_base;
        long long iused = 0;
        if ((long long)nbr + 2LL * E <= ints_free) {
            last = ip;
            last_base = lo;
            lvl = last + nbr;
            order = lvl + E;
            iused = (long long)nbr + 2LL * E;
        } else {
            last = A.b_last;
            last_base = 0;
            lvl = A.j_level + (size_t)j0 * JOINT_WAVE_ITERS;
            order = A.j_order + (size_t)j0 * JOINT_WAVE_ITERS;
        }
        for (int j = j0 + lane; j < j1; j += 32) {
            if (A.j_type[j] == 2) { if (A.j_a[j] >= 0) wake_body(A, A.j_a[j]); }
            else {
                if (A.j_a[j] >= 0) wake_body(A, A.j_a[j]);
                if (A.j_b[j] >= 0) wake_body(A, A.j_b[j]);
            }
            joint_prepare(A, j, rows ? rows + (size_t)(j - j0) * JD : &A.j_data[(size_t)j * JD]);
        }
        for (int i = lane; i < nbr; i += 32) last[lo + i - last_base] = -1;
        __syncwarp();
        const int D = waves ? warp_joint_levels(A, j0, J, iters, last, lvl, last_base)
                            : warp_levels(J, A.j_a + j0, A.j_b + j0, A.mtype, last, lvl, last_base);
        int *ls, *cur;
        if (iused > 0 && iused + 2LL * (D + 1) <= ints_free) {
            ls = ip + iused;
            cur = ls + D + 1;
        } else {
            ls = A.j_level_start + (size_t)j0 * JOINT_WAVE_ITERS + w;
            cur = A.j_level_start + ((size_t)A.NJ * JOINT_WAVE_ITERS + A.W + 1) + (size_t)j0 * JOINT_WAVE_ITERS + w;
        }
        // bucket the entries by level: ls[l] = first slot of level l
        for (int l = lane; l <= D; l += 32) ls[l] = 0;
        __syncwarp();
        for (int k = lane; k < E; k += 32)
            if (lvl[k] + 1 <= D) atomicAdd(&ls[lvl[k] + 1], 1);
        __syncwarp();
        warp_scan_inclusive(ls, D + 1);
        for (int l = lane; l <= D; l += 32) cur[l] = ls[l];
        __syncwarp();
        for (int k = lane; k < E; k += 32) {
            // a lone motor's entries carry bit 31: its iteration-0 entry runs all its iterations
            const bool alone = waves && motor_alone(A, j0 + k % J);
            order[atomicAdd(&cur[lvl[k]], 1)] = k | (alone ? (int)0x80000000u : 0);
        }
        if (V.s)
            for (int i = lane; i < nbr; i += 32)
                for (int q = 0; q < 3; q++) {
                    V.s[i * 6 + q] = A.v[(size_t)(lo + i) * 3 + q];
                    V.s[i * 6 + 3 + q] = A.w[(size_t)(lo + i) * 3 + q];
                }
        __syncwarp();
        const int rounds = waves ? 1 : iters;
        for (int it = 0; it < rounds; it++)
            for (int l = 0; l < D; l++) {
                const int qa = ls[l], qb = ls[l + 1];
                for (int q = qa + lane; q < qb; q += 32) {
                    const int v = order[q], e = v & 0x7FFFFFFF, jj = e % J, j = j0 + jj;
                    const double *Dr = rows ? rows + (size_t)jj * JD : &A.j_data[(size_t)j * JD];
                    if (v >= 0) joint_solve(A, j, Dr, V, dt);
                    else if (e < J) for (int k = 0; k < iters; k++) joint_solve(A, j, Dr, V, dt);
                }
                __syncwarp();
            }
        if (V.s)
            for (int i = lane; i < nbr; i += 32)
                if (A.mtype[lo + i] == 2)
                    for (int q = 0; q < 3; q++) {
                        A.v[(size_t)(lo + i) * 3 + q] = V.s[i * 6 + q];
                        A.w[(size_t)(lo + i) * 3 + q] = V.s[i * 6 + 3 + q];
                    }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// integrate positions (backend.py:42-49, mathutil.py:32-41,108-113) and
// island sleeping (world.py:510-567), one CTA per world
// ---------------------------------------------------------------------------
enum { BF_SLOW = 1, BF_READY = 2, BF_CONTACTED = 4, BF_NOTREADY = 8 };
enum { FIN_POSITIONS = 1, FIN_SLEEP = 2, FIN_COUNT = 4, FIN_GATED = 8 };

__device__ inline int uf_find(int *parent, int x) {
    volatile int *p = parent;
    while (true) {
        const int px = p[x];
        if (px == x) return x;
        const int gp = p[px];
        if (gp != px) p[x] = gp;
        x = px;
    }
}

__device__ inline void uf_union(int *parent, int a, int b) {
    while (true) {
        a = uf_find(parent, a);
        b = uf_find(parent, b);
        if (a == b) return;
        if (a > b) { const int t = a; a = b; b = t; }
        if (atomicCAS(&parent[b], b, a) == b) return;
    }
}

// Per body of the world: flags and union-find parents, in shared memory when
// the world has at most `cap` bodies (indices local to the world), else in
// the global arrays. Roots are each island's smallest index (uf_union links
// the larger root under the smaller), so labels do not depend on which of
// the two is used.
__global__ void k_finalize(Arena A, int mode, int cap) {
    extern __shared__ int fsm[];
    if ((mode & FIN_GATED) && overflowed(A)) return;
    if ((mode & FIN_COUNT) && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&A.status[ST_STEPS_DONE], 1);
    for (int wi = blockIdx.x; wi < A.W; wi += gridDim.x) {
        const int w = A.w_sched[wi];
        if (!A.w_active[w] || world_wide(A, w)) continue;
        const double dt = A.w_dt[w];
        const int b0 = A.w_body_off[w], nb = A.w_body_n[w], b1 = b0 + nb;
        if (mode & FIN_POSITIONS) {
            for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
                const int t = A.mtype[i];
                if (!((t == 2 || t == 1) && A.awake[i])) continue;
                double *p = &A.pos[i * 3], *q = &A.q[i * 4];
                const double *v = &A.v[i * 3], *om = &A.w[i * 3];
                for (int c = 0; c < 3; c++) p[c] = p[c] + v[c] * dt;
                const double ax = om[0], ay = om[1], az = om[2], aw = 0.0;
                const double bx = q[0], by = q[1], bz = q[2], bw = q[3];
                double m[4];
                m[0] = aw * bx + ax * bw + ay * bz - az * by;
                m[1] = aw * by - ax * bz + ay * bw + az * bx;
                m[2] = aw * bz + ax * by - ay * bx + az * bw;
                m[3] = aw * bw - ax * bx - ay * by - az * bz;
                double s[4];
                for (int c = 0; c < 4; c++) s[c] = q[c] + (0.5 * m[c]) * dt;
                const double n = sqrt(((s[0] * s[0] + s[1] * s[1]) + s[2] * s[2]) + s[3] * s[3]);
                const double d = np_max(n, 1e-12);
                for (int c = 0; c < 4; c++) q[c] = s[c] / d;
            }
        }
        if (!(mode & FIN_SLEEP)) continue;
        if (!(A.w_flags[w] & WF_SLEEP)) {
            for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) A.b_island[i] = -1;
            continue;
        }
        const bool local = nb <= cap;
        int *flag = local ? fsm : A.b_flag + b0;          // indexed by i - b0
        int *parent = local ? fsm + cap : A.b_parent + b0;
        __syncthreads();
        const double lin2 = 0.08 * 0.08, ang2 = 0.25 * 0.25;
        for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
            const bool dyn_i = A.mtype[i] == 2;
            const bool slow = dyn_i && speed2(&A.v[i * 3]) < lin2 && speed2(&A.w[i * 3]) < ang2;
            if (slow) A.timer[i] += dt; else A.timer[i] = 0.0;
            const bool ready = slow && A.timer[i] > 0.4;
            flag[i - b0] = (slow ? BF_SLOW : 0) | (ready ? BF_READY : 0);
            parent[i - b0] = i - b0;
        }
        __syncthreads();
        if (world_collides(A, w)) {
            int c0, c1;
            world_contacts(A, w, c0, c1);
            for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
                const int a = A.c_a[k], b = A.c_b[k];
                OMI_BOUNDS(A, a - b0, nb, BS_ISLAND_BODY, continue)
                OMI_BOUNDS(A, b - b0, nb, BS_ISLAND_BODY, continue)
                const bool da = A.mtype[a] == 2, db = A.mtype[b] == 2;
                if (da) atomicOr(&flag[a - b0], BF_CONTACTED);
                if (db) atomicOr(&flag[b - b0], BF_CONTACTED);
                if (da && db) uf_union(parent, a - b0, b - b0);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nb; i += blockDim.x) A.b_island[b0 + i] = b0 + uf_find(parent, i);
        __syncthreads();
        for (int i = threadIdx.x; i < nb; i += blockDim.x) {
            const int f = ((volatile int *)flag)[i];
            if ((f & BF_CONTACTED) && !(f & BF_READY)) atomicOr(&flag[A.b_island[b0 + i] - b0], BF_NOTREADY);
        }
        __syncthreads();
        for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
            const int f = ((volatile int *)flag)[i - b0];
            const bool dyn_i = A.mtype[i] == 2;
            bool to_sleep;
            if (f & BF_CONTACTED) to_sleep = !(((volatile int *)flag)[A.b_island[i] - b0] & BF_NOTREADY);
            else to_sleep = dyn_i && (f & BF_READY);
            if (!(f & BF_CONTACTED)) A.b_island[i] = -1;
            if (to_sleep) A.awake[i] = 0;
            if (dyn_i && !(f & BF_SLOW)) A.awake[i] = 1;
            if (!A.awake[i] && dyn_i) {
                for (int c = 0; c < 3; c++) { A.v[i * 3 + c] = 0.0; A.w[i * 3 + c] = 0.0; }
            }
        }
        __syncthreads();
    }
}

}  // namespace omi
