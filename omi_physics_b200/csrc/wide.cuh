// Wide worlds: the stages that run one block per world elsewhere (sort,
// sweep links, wake, contact sweep, warm-start cache store, positions and
// sleep) spread over many blocks for worlds large enough that one block (one
// SM) would bound the step. The results are the same bits as the
// one-block forms: the same arithmetic in the same dependency order.
//
// Launches carry the wide world's index in blockIdx.y (or as an argument for
// the sweep); x runs over the world's bodies, contacts or runs, grid-stride.
#pragma once
#include <cooperative_groups.h>

#include "kernels2.cuh"

namespace omi {

// per wide world, ints of global counters (zeroed before the solve stage)
constexpr int WIDE_STATE_INTS = 32;
enum { WS_HEAD = 0, WS_TAIL = 8, WS_CLAIMED = 16, WS_ABORT = 17, WS_HIST = 18, WS_CASCADE = 22, WS_SWEPT = 23 };
// set by the cluster sweep when it swept the world this step: the many-block
// sweep launched after it then has nothing to do
__device__ __forceinline__ bool wide_swept(const Arena &A, int wi) {
    return A.wide_state[wi * WIDE_STATE_INTS + WS_SWEPT] != 0;
}
// bodies per sort tile (sorted in shared memory, then merged in global memory)
constexpr int WSORT_TILE = 4096;
constexpr int WSORT_THREADS = 512;

__device__ __forceinline__ int wide_tid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int wide_stride() { return gridDim.x * blockDim.x; }

// ---------------------------------------------------------------------------
// sort (np.argsort(min_x, kind='stable'), broadphase.py:261): tiles sorted in
// shared memory by the merge sort of k_sort, then merged pairwise in global
// memory (each element placed by its rank in the partner run), then the
// sorted rows written as k_sort writes them
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(WSORT_THREADS) k_wsort_tiles(Arena A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = A.wide_w[blockIdx.y];
    if (!world_collides(A, w)) return;
    const int off = A.w_body_off[w], n = A.w_body_n[w];
    const int t0 = blockIdx.x * WSORT_TILE;
    if (t0 >= n) return;
    const int m = min(WSORT_TILE, n - t0);
    double *k0 = reinterpret_cast<double *>(smem), *k1 = k0 + WSORT_TILE;
    int *v0 = reinterpret_cast<int *>(k1 + WSORT_TILE), *v1 = v0 + WSORT_TILE;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        k0[i] = A.aabb_min[(off + t0 + i) * 3] + 0.0;      // -0.0 == 0.0; NaN stays NaN (sorts last)
        v0[i] = t0 + i;
    }
    __syncthreads();
    for (int width = 1; width < m; width <<= 1) {
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const int seg = (i / (2 * width)) * (2 * width);
            const int mid = min(seg + width, m), end = min(seg + 2 * width, m);
            const double key = k0[i];
            const int val = v0[i];
            int lo, hi, base;
            if (i < mid) { lo = mid; hi = end; base = i - seg; }
            else { lo = seg; hi = mid; base = i - mid; }
            const int start = lo;
            while (lo < hi) {
                const int q = (lo + hi) >> 1;
                if (key_less(k0[q], v0[q], key, val)) lo = q + 1; else hi = q;
            }
            const int pos = seg + base + (lo - start);
            k1[pos] = key;
            v1[pos] = val;
        }
        __syncthreads();
        double *tk = k0; k0 = k1; k1 = tk;
        int *tv = v0; v0 = v1; v1 = tv;
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        A.sort_k[0][off + t0 + i] = k0[i];
        A.sort_v[0][off + t0 + i] = v0[i];
    }
}

// one merge pass over runs of `width` elements: buffer src -> 1 - src
__global__ void k_wsort_merge(Arena A, int width, int src) {
    const int w = A.wide_w[blockIdx.y];
    if (!world_collides(A, w)) return;
    const int off = A.w_body_off[w], n = A.w_body_n[w];
    const double *ks = A.sort_k[src] + off;
    const int *vs = A.sort_v[src] + off;
    double *kd = A.sort_k[1 - src] + off;
    int *vd = A.sort_v[1 - src] + off;
    for (int i = wide_tid(); i < n; i += wide_stride()) {
        const int seg = (int)(((int64_t)i / (2 * (int64_t)width)) * 2 * width);
        const int mid = (int)min((int64_t)seg + width, (int64_t)n), end = (int)min((int64_t)seg + 2 * (int64_t)width, (int64_t)n);
        const double key = ks[i];
        const int val = vs[i];
        int lo, hi, base;
        if (i < mid) { lo = mid; hi = end; base = i - seg; }
        else { lo = seg; hi = mid; base = i - mid; }
        const int start = lo;
        while (lo < hi) {
            const int q = (lo + hi) >> 1;
            if (key_less(ks[q], vs[q], key, val)) lo = q + 1; else hi = q;
        }
        const int pos = seg + base + (lo - start);
        kd[pos] = key;
        vd[pos] = val;
    }
}

// the sorted rows of the step's broadphase, from buffer src (as k_sort<true>)
__global__ void k_wsort_rows(Arena A, int src) {
    const int w = A.wide_w[blockIdx.y];
    if (!world_collides(A, w)) return;
    const int off = A.w_body_off[w], n = A.w_body_n[w];
    for (int i = wide_tid(); i < n; i += wide_stride()) {
        const int body = off + A.sort_v[src][off + i];
        A.order[off + i] = body;
        A.sorted_x[off + i] = A.sort_k[src][off + i];
        double4 *row = reinterpret_cast<double4 *>(&A.srt_box[(size_t)(off + i) * 8]);
        const double *lo = &A.aabb_min[body * 3], *hi = &A.aabb_max[body * 3];
        row[0] = make_double4(lo[0], hi[0], lo[1], hi[1]);
        row[1] = make_double4(lo[2], hi[2], 0.0, 0.0);
        const bool sensor = A.tshape[body] >= 0;
        A.srt_info[off + i] = A.mtype[body] | (A.shape[body] >= 0 && !sensor ? 4 : 0) |
                              (A.awake[body] ? 8 : 0) | (sensor ? 16 : 0) | (A.filter_row[body] << 5);
    }
}

// ---------------------------------------------------------------------------
// wake (_wake_sleepers, solver.py:321-337): phase 0 looks for a sleeper moving
// faster than the wake threshold among the contacts (then the pass must run
// in contact order: one thread does it); phase 1 wakes, in parallel when no
// woken body can wake another (as k_wake decides per world)
// ---------------------------------------------------------------------------
__global__ void k_wwake(Arena A, int phase) {
    if (overflowed(A)) return;
    const int wi = blockIdx.y, w = A.wide_w[wi];
    if (!world_collides(A, w)) return;
    int c0, c1;
    world_contacts(A, w, c0, c1);
    int *st = A.wide_state + wi * WIDE_STATE_INTS;
    const double thr = 0.15 * 0.15;
    if (phase == 0) {
        bool cascade = false;
        for (int k = c0 + wide_tid(); k < c1; k += wide_stride()) {
            const int e[2] = {A.c_a[k], A.c_b[k]};
            for (int j = 0; j < 2; j++) {
                const int x = e[j];
                cascade |= A.mtype[x] == 2 && !A.awake[x] && speed2(&A.v[x * 3]) > thr;
            }
        }
        if (__syncthreads_or(cascade) && threadIdx.x == 0) atomicOr(&st[WS_CASCADE], 1);
        return;
    }
    if (*(volatile int *)&st[WS_CASCADE]) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
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
        return;
    }
    for (int k = c0 + wide_tid(); k < c1; k += wide_stride()) {
        const int a = A.c_a[k], b = A.c_b[k];
        const int ta = A.mtype[a], tb = A.mtype[b];
        if (!A.awake[b] && (ta == 1 || (ta == 2 && A.awake[a] && speed2(&A.v[a * 3]) > thr))) wake_body(A, b);
        if (!A.awake[a] && (tb == 1 || (tb == 2 && A.awake[b] && speed2(&A.v[b * 3]) > thr))) wake_body(A, a);
    }
}

// ---------------------------------------------------------------------------
// sweep links (k_levels' runs, buckets and predecessor / successor codes) in
// five grid passes and two scans:
//   k_wl_flags  per contact: starts a run? (wide worlds only); zero buckets
//   (scan of the flags over all contacts)
//   k_wl_runs   per run start: run_k, run_a, run_b; per wide world: w_runs
//   k_wl_count  per run: run_n, bucket counts of its dynamic bodies
//   (scan of the counts over all bodies)
//   k_wl_fill   per run: its index into both bodies' buckets
//   k_wl_links  per run: predecessor / successor codes, run_kn, run_need
// ---------------------------------------------------------------------------
__global__ void k_wl_flags(Arena A) {
    if (overflowed(A)) return;
    const int Ktot = A.contact_scan[A.pair_scan[A.NB]];
    if (blockIdx.x == 0 && threadIdx.x == 0) *A.k_total = Ktot;
    for (int k = wide_tid(); k < Ktot; k += wide_stride()) {
        const int a = A.c_a[k], b = A.c_b[k];
        const int w = A.body_world[a];
        int start = 0;
        if (world_wide(A, w) && world_collides(A, w)) {
            int c0, c1;
            world_contacts(A, w, c0, c1);
            start = k == c0 || a != A.c_a[k - 1] || b != A.c_b[k - 1];
            if (!start && (A.kind[a] == 5 || A.kind[b] == 5))
                start = A.c_n[k * 3] != A.c_n[k * 3 - 3] || A.c_n[k * 3 + 1] != A.c_n[k * 3 - 2] ||
                        A.c_n[k * 3 + 2] != A.c_n[k * 3 - 1];
        }
        A.wl_flag[k] = start;
    }
    for (int i = wide_tid(); i < A.NB; i += wide_stride()) A.wl_cnt[i] = 0;
}

__global__ void k_wl_runs(Arena A) {
    if (overflowed(A)) return;
    const int Ktot = A.contact_scan[A.pair_scan[A.NB]];
    for (int k = wide_tid(); k < Ktot; k += wide_stride()) {
        if (!A.wl_flag[k]) continue;
        const int a = A.c_a[k], b = A.c_b[k];
        const int w = A.body_world[a];
        int c0, c1;
        world_contacts(A, w, c0, c1);
        const int r = A.wl_scan[k] - A.wl_scan[c0];
        A.run_k[c0 + r] = k - c0;
        A.run_a[c0 + r] = A.mtype[a] == 2 ? a : -1;
        A.run_b[c0 + r] = A.mtype[b] == 2 ? b : -1;
    }
    for (int wi = wide_tid(); wi < A.n_wide; wi += wide_stride()) {
        const int w = A.wide_w[wi];
        if (!world_collides(A, w)) continue;
        int c0, c1;
        world_contacts(A, w, c0, c1);
        const int K = c1 - c0;
        A.w_runs[w] = K ? A.wl_scan[c1] - A.wl_scan[c0] : 0;
        if (K >= (1 << 24)) {                      // run_kn packs contact offsets in 24 bits
            A.w_runs[w] = 0;
            atomicOr(&A.status[ST_SWEEP_TIMEOUT], 1);
        }
    }
}

__global__ void k_wl_count(Arena A) {
    if (overflowed(A)) return;
    const int w = A.wide_w[blockIdx.y];
    if (!world_collides(A, w)) return;
    int c0, c1;
    world_contacts(A, w, c0, c1);
    const int K = c1 - c0, R = A.w_runs[w];
    for (int r = wide_tid(); r < R; r += wide_stride()) {
        const int end = r + 1 < R ? A.run_k[c0 + r + 1] : K;
        A.run_n[c0 + r] = end - A.run_k[c0 + r];
        const int a = A.run_a[c0 + r], b = A.run_b[c0 + r];
        if (a >= 0) atomicAdd(&A.wl_cnt[a], 1);
        if (b >= 0) atomicAdd(&A.wl_cnt[b], 1);
    }
}

__global__ void k_wl_fill(Arena A) {
    if (overflowed(A)) return;
    const int w = A.wide_w[blockIdx.y];
    if (!world_collides(A, w)) return;
    int c0, c1;
    world_contacts(A, w, c0, c1);
    const int R = A.w_runs[w];
    for (int r = wide_tid(); r < R; r += wide_stride()) {
        const int a = A.run_a[c0 + r], b = A.run_b[c0 + r];
        // counts go back down to zero as the slots are taken (bucket order does not matter)
        if (a >= 0) A.wl_list[A.wl_bstart[a] + atomicSub(&A.wl_cnt[a], 1) - 1] = r;
        if (b >= 0) A.wl_list[A.wl_bstart[b] + atomicSub(&A.wl_cnt[b], 1) - 1] = r;
    }
}

__global__ void k_wl_links(Arena A) {
    if (overflowed(A)) return;
    const int w = A.wide_w[blockIdx.y];
    if (!world_collides(A, w)) return;
    int c0, c1;
    world_contacts(A, w, c0, c1);
    const int R = A.w_runs[w];
    for (int r = wide_tid(); r < R; r += wide_stride()) {
        const int a = A.run_a[c0 + r], b = A.run_b[c0 + r];
        int pa = LEVEL_NONE, pb = LEVEL_NONE, sa = LEVEL_NONE, sb = LEVEL_NONE;
        if (a >= 0) run_link_codes(A.wl_list, A.wl_bstart[a], A.wl_bstart[a + 1], r, pa, sa);
        if (b >= 0) run_link_codes(A.wl_list, A.wl_bstart[b], A.wl_bstart[b + 1], r, pb, sb);
        A.run_pa[c0 + r] = pa;
        A.run_pb[c0 + r] = pb;
        A.run_sa[c0 + r] = sa;
        A.run_sb[c0 + r] = sb;
        A.run_kn[c0 + r] = A.run_k[c0 + r] | (A.run_n[c0 + r] << 24);
        // (the test hook's run asks for 3 same-pass arrivals of at most 2: it never becomes ready)
        A.run_need[c0 + r] = ((pa >= 0) + (pb >= 0)) | (((pa != LEVEL_NONE) + (pb != LEVEL_NONE)) << 2) |
                             (r == A.stall_run ? 3 : 0);
    }
}

// ---------------------------------------------------------------------------
// the contact sweep of one wide world on many blocks: the dataflow of
// k_iterate's sweep_world (same entries, same predecessor counts, same
// per-class rings) with its state in global memory - arrival counts, the
// ring and the ring counters - and device-scope release / acquire in place of
// block scope. Velocities, positions and impulses stay in their global
// arrays. A block claims only published entries, so the blocks need not all
// be resident at once. Every wait is
// bounded by Arena::spin_limit; a wait that runs out sets the world's abort
// flag, which ends every other wait, and ST_SWEEP_TIMEOUT. The roots are
// published by a launch of their own (k_wsweep_seed), so no block waits on
// work that only another block could start: with several groups' sweeps on
// the GPU at once, whichever blocks are resident make progress. A thread
// whose arrival makes a successor ready runs that successor next itself
// (counted as claimed) and publishes only a second one: a chain of entries
// then skips the ring's publish, poll, claim and slot read between its
// links, four to five device-memory round trips each (the hull pile's late
// sweep: 7.8 -> 6.3 ms at 72K runs).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_gpu(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int *p, int v) {
    asm volatile("st.release.gpu.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// the ring of a wide world: per class its slot count and first slot
struct WideRings {
    int size[SWEEP_CLASSES], base[SWEEP_CLASSES];
};

__device__ __forceinline__ void wide_push(int *ring, int *st, const WideRings &wr, int e, int n) {
    const int c = entry_class(e >> PASS_SHIFT, n, true);
    const int pos = atomicAdd(&st[WS_TAIL + c], 1);
    if (pos >= wr.size[c]) { atomicExch(&st[WS_ABORT], 1); return; }   // never with a consistent graph
    st_release_gpu(&ring[wr.base[c] + pos], e + 1);
}

// arrival counts zeroed, ring cleared, runs counted by length (for the class sizes)
__global__ void k_wsweep_init(Arena A, int wi) {
    __shared__ int hist[4];
    if (overflowed(A) || wide_swept(A, wi)) return;
    const int w = A.wide_w[wi];
    if (!world_collides(A, w)) return;
    int c0, c1;
    world_contacts(A, w, c0, c1);
    const int R = A.w_runs[w], N = world_passes(A, w) * R;
    if (threadIdx.x < 4) hist[threadIdx.x] = 0;
    __syncthreads();
    for (int r = wide_tid(); r < R; r += wide_stride()) {
        A.run_done[c0 + r] = 0;
        atomicAdd(&hist[min(A.run_kn[c0 + r] >> 24, 4) - 1], 1);
    }
    int *ring = A.c_order + (size_t)c0 * A.max_passes;
    for (int e = wide_tid(); e < N; e += wide_stride()) ring[e] = 0;
    __syncthreads();
    if (threadIdx.x < 4 && hist[threadIdx.x])
        atomicAdd(&A.wide_state[wi * WIDE_STATE_INTS + WS_HIST + threadIdx.x], hist[threadIdx.x]);
}

// per class: slots and first slot of the ring (class = (pass 0 ? 4 : 0) +
// min(run length, 4) - 1), from the run-length counts of k_wsweep_init
__device__ __forceinline__ void wide_rings(const int *st, int P, WideRings &wr) {
    int acc = 0;
    for (int c = 0; c < SWEEP_CLASSES; c++) {
        const int cnt = st[WS_HIST + (c & 3)];
        wr.size[c] = c >= 4 ? cnt : cnt * (P - 1);
        wr.base[c] = acc;
        acc += wr.size[c];
    }
}

// the entries with no predecessor - pass-0 runs that start both bodies'
// chains - published before the sweep starts, so that no block of the sweep
// depends on another block having started
__global__ void k_wsweep_seed(Arena A, int wi) {
    __shared__ WideRings wr;
    if (overflowed(A) || wide_swept(A, wi)) return;
    const int w = A.wide_w[wi];
    if (!world_collides(A, w)) return;
    int *st = A.wide_state + wi * WIDE_STATE_INTS;
    const int R = A.w_runs[w];
    int c0, c1;
    world_contacts(A, w, c0, c1);
    if (threadIdx.x == 0) wide_rings(st, world_passes(A, w), wr);
    __syncthreads();
    int *ring = A.c_order + (size_t)c0 * A.max_passes;
    for (int r = wide_tid(); r < R; r += wide_stride())
        if ((A.run_need[c0 + r] & 3) == 0) wide_push(ring, st, wr, r, A.run_kn[c0 + r] >> 24);
}

__global__ void __launch_bounds__(SWEEP_THREADS) k_wsweep(Arena A, int wi) {
    __shared__ WideRings wr;
    if (overflowed(A) || wide_swept(A, wi)) return;
    const int w = A.wide_w[wi];
    if (!world_collides(A, w)) return;
    int *st = A.wide_state + wi * WIDE_STATE_INTS;
    const int R = A.w_runs[w];
    if (R == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) A.w_levels[w] = 0;
        return;
    }
    int c0, c1;
    world_contacts(A, w, c0, c1);
    const int P = world_passes(A, w);
    const int N = P * R;
    if (threadIdx.x == 0) wide_rings(st, P, wr);
    __syncthreads();
    int *ring = A.c_order + (size_t)c0 * A.max_passes;
    int *arrived = A.run_done + c0;
    const int *run_kn = A.run_kn + c0, *run_need = A.run_need + c0;
    const int *run_sa = A.run_sa + c0, *run_sb = A.run_sb + c0;
    const bool warm = (A.w_flags[w] & WF_WARM) != 0;
    const bool vel = warm || A.w_iters[w] > 0;
    const double slop = A.w_solver[w * 2 + 1];
    VelView V;
    V.s = nullptr;
    V.b0 = A.w_body_off[w];
    ImpView I;
    I.s = nullptr;
    I.c0 = c0;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int lo = 0, cnt = 0;
        if (lane == 0) {
            const int first = ((threadIdx.x >> 5) + blockIdx.x) & (SWEEP_CLASSES - 1);
            int idle = 0;
            for (int it = 0;; it++) {
                if (ld_relaxed_gpu(&st[WS_CLAIMED]) >= N || ld_relaxed_gpu(&st[WS_ABORT])) { cnt = -1; break; }
                bool got = false;
                for (int j = 0; j < SWEEP_CLASSES && !got; j++) {
                    const int c = (first + j) & (SWEEP_CLASSES - 1);
                    const int h = ld_relaxed_gpu(&st[WS_HEAD + c]);
                    const int t = min(ld_relaxed_gpu(&st[WS_TAIL + c]), wr.size[c]);
                    if (t > h) {
                        const int want = min(t - h, A.sweep_claim);
                        if (atomicCAS(&st[WS_HEAD + c], h, h + want) == h) {
                            atomicAdd(&st[WS_CLAIMED], want);
                            lo = wr.base[c] + h;
                            cnt = want;
                            got = true;
                        }
                    }
                }
                if (got) break;
                if (it >= A.spin_limit) { atomicExch(&st[WS_ABORT], 1); cnt = -1; break; }
                __nanosleep(min(32 << min(idle++, 5), 1024));      // back off while nothing is ready
            }
        }
        cnt = __shfl_sync(FULL, cnt, 0);
        lo = __shfl_sync(FULL, lo, 0);
        if (cnt < 0) break;
        if (lane < cnt) {
            int e1 = 0;
            for (int it = 0; it < A.spin_limit; it++) {   // the pusher is between its two steps
                e1 = ld_acquire_gpu(&ring[lo + lane]);
                if (e1 || ld_relaxed_gpu(&st[WS_ABORT])) break;
            }
            if (e1 == 0) atomicExch(&st[WS_ABORT], 1);
            else {
                int e = e1 - 1;
                for (int hop = 0; e >= 0; hop++) {
                    const int r = e & PASS_MASK, p = e >> PASS_SHIFT;
                    const int v = __ldg(run_kn + r);
                    const int k0 = c0 + (v & 0xFFFFFF), n = v >> 24;
                    double row0[CD];
                    load_row(A, k0, row0);
                    const int sa = __ldg(run_sa + r), sb = __ldg(run_sb + r);
#ifdef OMI_BOUNDS_CHECK
                    if (sweep_rows_ok(A, row0, V.b0, A.w_body_n[w]))
#endif
                    run_pass(A, V, I, row0, k0, n, vel, warm && p == 0, p == 0, slop);
                    // release this entry's writes, then count into the successors
                    fence_acq_rel_gpu();
                    const int sides[2] = {sa, sb};
                    int next = -1;
#pragma unroll
                    for (int sd = 0; sd < 2; sd++) {
                        const int sc = sides[sd];
                        int ps, rs;
                        if (sc >= 0) { ps = p; rs = sc; }
                        else if (sc != LEVEL_NONE && p + 1 < P) { ps = p + 1; rs = -sc - 1; }
                        else continue;
                        OMI_BOUNDS(A, rs, R, BS_SWEEP_RUN, continue)
                        if (atomicAdd(&arrived[rs], 1) + 1 == need_of(__ldg(run_need + rs), ps)) {
                            fence_acq_rel_gpu();             // acquire the other arrivals' writes
                            if (next < 0) { next = (ps << PASS_SHIFT) | rs; continue; }
                            wide_push(ring, st, wr, (ps << PASS_SHIFT) | rs, __ldg(run_kn + rs) >> 24);
                        }
                    }
                    // a successor this entry made ready runs next on this thread,
                    // counted as claimed, instead of going through the ring
                    if (next >= 0) {
                        atomicAdd(&st[WS_CLAIMED], 1);
                        if ((hop & 15) == 15 && ld_relaxed_gpu(&st[WS_ABORT])) break;
                    }
                    e = next;
                }
            }
        }
        __syncwarp();
    }
    if (lane == 0 && ld_relaxed_gpu(&st[WS_ABORT])) atomicOr(&A.status[ST_SWEEP_TIMEOUT], 1);
    if (blockIdx.x == 0 && threadIdx.x == 0) A.w_levels[w] = -2;     // not tracked on the many-block sweep
}

// the sweep of wide world blockIdx.x by one block: k_iterate's sweep_world on
// the tables the wide links wrote (the same format as k_levels')
__global__ void __launch_bounds__(SWEEP_THREADS) k_wsweep_one(Arena A, int smem_doubles) {
    extern __shared__ __align__(16) double smem_d[];
    __shared__ SweepShared sh;
    if (overflowed(A)) return;
    const int w = A.wide_w[blockIdx.x];
    if (!world_collides(A, w)) return;
    sweep_world(A, w, smem_d, smem_doubles, threadIdx.x, SWEEP_THREADS, 0, sh);
}

// ---------------------------------------------------------------------------
// The contact sweep of one wide world on one thread-block cluster of C CTAs
// (co-scheduled by the hardware, so every CTA of it is resident). The runs
// are split into C contiguous ranges (contacts come in pair order, so a range
// is a slab of the world); CTA b owns the entries of its range: their arrival
// counts and work ring live in its shared memory (or, when they do not fit,
// in the world's global slices of them) and only its warps claim them. An
// entry whose last predecessor finishes in another CTA is counted and
// published through distributed shared memory with cluster-scope release /
// acquire; everything else stays CTA-local. The dataflow - entries, their
// predecessor counts, the per-class rings - is k_iterate's, so the results
// are the same bits. Velocities, positions and impulses stay in global
// memory. Waits are bounded as in k_wsweep.
// ---------------------------------------------------------------------------
namespace cg = cooperative_groups;

struct ClusterShared {
    int head[SWEEP_CLASSES], tail[SWEEP_CLASSES], size[SWEEP_CLASSES], base[SWEEP_CLASSES];
    int hist[4];
    int claimed, abort, n_owned, fit, staged, imp_staged;
};

__device__ __forceinline__ int ld_acquire_cluster(const int *p) {
    int v;
    asm volatile("ld.acquire.cluster.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_cluster(int *p, int v) {
    asm volatile("st.release.cluster.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_cluster() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }

// the CTA owning run r of R, and the first run of CTA b, for C CTAs
__device__ __forceinline__ int cl_home(int r, int R, int C) { return (int)(((long long)r * C) / R); }
__device__ __forceinline__ int cl_first(int b, int R, int C) { return (int)(((long long)b * R + C - 1) / C); }

// Shared memory of CTA h (ints; rb = its runs): arrival counts (rb), work
// ring (P * rb), the slots of each run's two bodies (2 * rb), the bodies it
// owns (2 * rb at most: a body is owned by the CTA of its first run), its
// runs' tables (CL_TAB * rb: packed first contact and count, need counts,
// the two successor codes, and whether a predecessor lies in another CTA),
// then, 8-byte aligned, the owned bodies' records - v (3), w (3), pos (3) -
// and, when room is left, the impulses of its contacts.
constexpr int CL_REC = 9;
constexpr int CL_TAB = 5;
enum { CT_KN = 0, CT_NEED = 1, CT_SA = 2, CT_SB = 3, CT_XPRED = 4 };
__device__ __forceinline__ int cl_tab_off(int rb, int P) { return rb * (1 + P + 2 + 2); }
__device__ __forceinline__ int cl_ints(int rb, int P) { return rb * (1 + P + 2 + 2 + CL_TAB); }
__device__ __forceinline__ int cl_rec_off(int rb, int P) { return (cl_ints(rb, P) + 1) & ~1; }   // in ints

// where CTA h keeps its arrival counts and ring (its shared memory when the
// tables fit, else the world's global slices of them)
struct ClusterHome {
    int *arrived;    // indexed by run - first run of h
    int *ring;
};

template <int C>
__device__ __forceinline__ ClusterHome cl_home_arrays(const Arena &A, cg::cluster_group &cluster, int *csm, int h,
                                                      int R, int P, int c0, int smem_ints, int me) {
    const int r0 = cl_first(h, R, C), rb = cl_first(h + 1, R, C) - r0;
    ClusterHome H;
    if ((long long)cl_ints(rb, P) <= smem_ints) {
        int *base = h == me ? csm : cluster.map_shared_rank(csm, h);
        H.arrived = base;
        H.ring = base + rb;
    } else {
        H.arrived = A.run_done + c0 + r0;
        H.ring = A.c_order + (size_t)c0 * A.max_passes + (size_t)P * r0;
    }
    return H;
}

// run_pass on staged bodies: ra / rb are the bodies' records (v, w, pos) in
// their owners' shared memory, or nullptr for a body that is not dynamic
// (read from the global arrays, never written)
__device__ __forceinline__ void run_pass_rec(const Arena &A, double *ra, double *rb, const ImpView &I,
                                             const double *row0, int k0, int n, bool vel, bool warm_pass,
                                             bool pos_pass, double slop) {
    PairRow r;
    load_pair(row0, r);
    PairVel s;
    double pa[3], pb[3];
    for (int q = 0; q < 3; q++) {
        s.la[q] = ra ? ra[q] : A.v[r.a * 3 + q];
        s.aa[q] = ra ? ra[3 + q] : A.w[r.a * 3 + q];
        s.lb[q] = rb ? rb[q] : A.v[r.b * 3 + q];
        s.ab[q] = rb ? rb[3 + q] : A.w[r.b * 3 + q];
    }
    if (pos_pass)
        for (int q = 0; q < 3; q++) {
            pa[q] = ra ? ra[6 + q] : A.pos[r.a * 3 + q];
            pb[q] = rb ? rb[6 + q] : A.pos[r.b * 3 + q];
        }
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
    if (r.da) for (int q = 0; q < 3; q++) { ra[q] = s.la[q]; ra[3 + q] = s.aa[q]; }
    if (r.db) for (int q = 0; q < 3; q++) { rb[q] = s.lb[q]; rb[3 + q] = s.ab[q]; }
    if (pos_pass) {
        if (r.da) for (int q = 0; q < 3; q++) ra[6 + q] = pa[q];
        if (r.db) for (int q = 0; q < 3; q++) rb[6 + q] = pb[q];
    }
}

// The sweep on one cluster. Bodies: when every CTA's share fits (the
// cluster agrees on it), each dynamic body's record lives in the shared
// memory of the CTA of its first run and the others reach it through
// distributed shared memory; otherwise records are the global arrays.
// A CTA whose successors and written records are all its own releases with
// a CTA-scope fence, else cluster scope.
// With `handoff`, a world whose records do not fit is left to the many-block
// sweep launched after this kernel (on 16 SMs with every record and table in
// global memory the cluster is slower than that sweep on 32: a hull pile of
// 32768 bodies at 72K runs takes 13.4 ms here against 8.3 ms there); a world
// the cluster sweeps is marked WS_SWEPT, which ends the many-block launches.
template <int C>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(SWEEP_THREADS) k_csweep(Arena A, int wi, int smem_ints,
                                                                                   int handoff) {
    extern __shared__ __align__(16) int csm[];
    __shared__ ClusterShared cs;
    cg::cluster_group cluster = cg::this_cluster();
    // every CTA takes the same early exits (they read the same words), so all
    // or none reach the cluster barriers below
    if (overflowed(A)) return;
    const int w = A.wide_w[wi];
    if (!world_collides(A, w)) return;
    const int R = A.w_runs[w];
    if (R == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) A.w_levels[w] = 0;
        return;
    }
    const int me = (int)cluster.block_rank();
    int c0, c1;
    world_contacts(A, w, c0, c1);
    const int K = c1 - c0;
    const int P = world_passes(A, w);
    const int r0 = cl_first(me, R, C), Rb = cl_first(me + 1, R, C) - r0;
    const int Nb = P * Rb;
    int *gabort = &A.wide_state[wi * WIDE_STATE_INTS + WS_ABORT];
    int *slotmap = A.wl_cnt;                      // per body: owner << 20 | slot (free after the links)
    const int *run_kn = A.run_kn + c0, *run_need = A.run_need + c0;
    const int *run_sa = A.run_sa + c0, *run_sb = A.run_sb + c0;
    const ClusterHome mine = cl_home_arrays<C>(A, cluster, csm, me, R, P, c0, smem_ints, me);
    const bool tables_local = cl_ints(Rb, P) <= smem_ints;
    int *rslot = csm + Rb * (1 + P);              // (when tables_local) 2 per run
    int *owned = rslot + 2 * Rb;                  // (when tables_local) owned bodies
    double *recs = reinterpret_cast<double *>(csm + cl_rec_off(Rb, P));
    if (threadIdx.x < SWEEP_CLASSES) { cs.head[threadIdx.x] = 0; cs.tail[threadIdx.x] = 0; }
    if (threadIdx.x < 4) cs.hist[threadIdx.x] = 0;
    if (threadIdx.x == 0) { cs.claimed = 0; cs.abort = 0; cs.n_owned = 0; }
    __syncthreads();
    int *rtab = csm + cl_tab_off(Rb, P);         // (when tables_local) CL_TAB per run
    for (int i = threadIdx.x; i < Rb; i += blockDim.x) {
        const int r = r0 + i;
        mine.arrived[i] = 0;
        atomicAdd(&cs.hist[min(run_kn[r] >> 24, 4) - 1], 1);
        if (!tables_local) continue;
        {
            int *t = rtab + CL_TAB * i;
            t[CT_KN] = run_kn[r];
            t[CT_NEED] = run_need[r];
            t[CT_SA] = run_sa[r];
            t[CT_SB] = run_sb[r];
            int x = 0;
            const int pc[2] = {A.run_pa[c0 + r], A.run_pb[c0 + r]};
            for (int q = 0; q < 2; q++)
                if (pc[q] != LEVEL_NONE) x |= cl_home(pc[q] >= 0 ? pc[q] : -pc[q] - 1, R, C) != me;
            t[CT_XPRED] = x;
        }
        // a body belongs to the CTA of its first run (whose predecessor code points to the previous pass)
        const int a = A.run_a[c0 + r], b = A.run_b[c0 + r];
        const int pa = A.run_pa[c0 + r], pb = A.run_pb[c0 + r];
        if (a >= 0 && pa < 0 && pa != LEVEL_NONE) {
            const int sl = atomicAdd(&cs.n_owned, 1);
            owned[sl] = a;
            slotmap[a] = (me << 20) | sl;
        }
        if (b >= 0 && pb < 0 && pb != LEVEL_NONE) {
            const int sl = atomicAdd(&cs.n_owned, 1);
            owned[sl] = b;
            slotmap[b] = (me << 20) | sl;
        }
    }
    for (int e = threadIdx.x; e < Nb; e += blockDim.x) mine.ring[e] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int c = 0; c < SWEEP_CLASSES; c++) {
            const int cnt = cs.hist[c & 3];
            cs.size[c] = c >= 4 ? cnt : cnt * (P - 1);
            cs.base[c] = acc;
            acc += cs.size[c];
        }
        cs.fit = tables_local && (long long)cl_rec_off(Rb, P) + 2LL * CL_REC * cs.n_owned <= smem_ints;
    }
    __threadfence();
    cluster.sync();               // rings, counts, ownership and fit flags ready cluster-wide
    if (threadIdx.x == 0) {
        int all = 1;
        for (int h = 0; h < C; h++) all &= cluster.map_shared_rank(&cs, h)->fit;
        cs.staged = all;
    }
    __syncthreads();
    const bool staged = cs.staged != 0;
    if (handoff) {
        // every CTA reads the same flags, so all leave here or none; the
        // barrier keeps each CTA's shared memory alive until every other has
        // read its fit flag
        if (!staged) {
            cluster.sync();
            return;
        }
        if (me == 0 && threadIdx.x == 0) A.wide_state[wi * WIDE_STATE_INTS + WS_SWEPT] = 1;
    }
    // impulses of this CTA's contacts (a contiguous range: its runs') in shared memory when room is left
    const int k_lo = Rb ? (run_kn[r0] & 0xFFFFFF) : 0;
    const int k_hi = Rb ? (r0 + Rb < R ? (run_kn[r0 + Rb] & 0xFFFFFF) : K) : 0;
    ImpView I;
    I.s = nullptr;
    I.c0 = c0 + k_lo;
    if (staged) {
        for (int i = threadIdx.x; i < cs.n_owned; i += blockDim.x) {
            const int body = owned[i];
            double *rec = recs + (size_t)i * CL_REC;
            for (int q = 0; q < 3; q++) {
                rec[q] = A.v[body * 3 + q];
                rec[3 + q] = A.w[body * 3 + q];
                rec[6 + q] = A.pos[body * 3 + q];
            }
        }
        for (int i = threadIdx.x; i < Rb; i += blockDim.x) {
            const int a = A.run_a[c0 + r0 + i], b = A.run_b[c0 + r0 + i];
            rslot[2 * i] = a >= 0 ? slotmap[a] : -1;
            rslot[2 * i + 1] = b >= 0 ? slotmap[b] : -1;
        }
        const long long imp_off = ((long long)cl_rec_off(Rb, P) + 2LL * CL_REC * cs.n_owned + 3) & ~3LL;
        if (imp_off + 2LL * 3 * (k_hi - k_lo) <= smem_ints) {
            I.s = reinterpret_cast<double *>(csm + imp_off);
            for (int i = threadIdx.x; i < 3 * (k_hi - k_lo); i += blockDim.x) I.s[i] = A.c_imp[(c0 + k_lo) * 3 + i];
        }
    }
    __syncthreads();
    cluster.sync();               // every record staged before any CTA reaches another's
    const bool warm = (A.w_flags[w] & WF_WARM) != 0;
    const bool vel = warm || A.w_iters[w] > 0;
    const double slop = A.w_solver[w * 2 + 1];
    VelView V;
    V.s = nullptr;
    V.b0 = A.w_body_off[w];
    // run rs's table row in its home CTA (DSMEM when remote); nullptr when the
    // home's tables are not in shared memory
    auto tab_of = [&](int rs) -> const int * {
        const int h = cl_home(rs, R, C);
        const int h0 = cl_first(h, R, C), hr = cl_first(h + 1, R, C) - h0;
        if ((long long)cl_ints(hr, P) > smem_ints) return nullptr;
        const int *base = (h == me ? csm : cluster.map_shared_rank(csm, h)) + cl_tab_off(hr, P);
        return base + CL_TAB * (rs - h0);
    };
    // the record of a staged body in its owner's shared memory
    auto rec_of = [&](int slot) -> double * {
        if (slot < 0) return nullptr;
        const int h = slot >> 20;
        const int hr = cl_first(h + 1, R, C) - cl_first(h, R, C);
        double *base = reinterpret_cast<double *>((h == me ? csm : cluster.map_shared_rank(csm, h)) + cl_rec_off(hr, P));
        return base + (size_t)(slot & 0xFFFFF) * CL_REC;
    };
    // publish entry e (run rs of pass ps, run length n) to its home's ring
    auto push = [&](int e, int rs, int n) {
        const int h = cl_home(rs, R, C);
        ClusterShared *hs = h == me ? &cs : cluster.map_shared_rank(&cs, h);
        const ClusterHome H = h == me ? mine : cl_home_arrays<C>(A, cluster, csm, h, R, P, c0, smem_ints, me);
        const int c = entry_class(e >> PASS_SHIFT, n, true);
        const int pos = atomicAdd(&hs->tail[c], 1);
        if (pos >= hs->size[c]) { cs.abort = 1; atomicExch(gabort, 1); return; }   // never with a consistent graph
        if (h == me) st_release_cta(&H.ring[hs->base[c] + pos], e + 1);
        else st_release_cluster(&H.ring[hs->base[c] + pos], e + 1);
    };
    for (int r = r0 + (int)threadIdx.x; r < r0 + Rb; r += blockDim.x)
        if ((__ldg(run_need + r) & 3) == 0) push(r, r, __ldg(run_kn + r) >> 24);
    const int lane = threadIdx.x & 31;
    for (;;) {
        int lo = 0, cnt = 0;
        if (lane == 0) {
            const int first = (threadIdx.x >> 5) & (SWEEP_CLASSES - 1);
            for (int it = 0;; it++) {
                if (*(volatile int *)&cs.claimed >= Nb || *(volatile int *)&cs.abort) { cnt = -1; break; }
                bool got = false;
                for (int j = 0; j < SWEEP_CLASSES && !got; j++) {
                    const int c = (first + j) & (SWEEP_CLASSES - 1);
                    const int h = *(volatile int *)&cs.head[c];
                    const int t = min(*(volatile int *)&cs.tail[c], cs.size[c]);
                    if (t > h) {
                        const int want = min(t - h, A.sweep_claim);
                        if (atomicCAS(&cs.head[c], h, h + want) == h) {
                            atomicAdd(&cs.claimed, want);
                            lo = cs.base[c] + h;
                            cnt = want;
                            got = true;
                        }
                    }
                }
                if (got) break;
                if (it >= A.spin_limit) { cs.abort = 1; atomicExch(gabort, 1); cnt = -1; break; }
                if ((it & 255) == 255 && ld_relaxed_gpu(gabort)) { cs.abort = 1; cnt = -1; break; }
                __nanosleep(32);
            }
        }
        cnt = __shfl_sync(FULL, cnt, 0);
        lo = __shfl_sync(FULL, lo, 0);
        if (cnt < 0) break;
        if (lane < cnt) {
            int e1 = 0;
            for (int it = 0; it < A.spin_limit; it++) {   // the pusher is between its two steps
                e1 = ld_acquire_cluster(&mine.ring[lo + lane]);
                if (e1 || *(volatile int *)&cs.abort) break;
            }
            if (e1 == 0) { cs.abort = 1; atomicExch(gabort, 1); }
            else {
                const int e = e1 - 1;
                const int r = e & PASS_MASK, p = e >> PASS_SHIFT;
                const int *tr = tables_local ? rtab + CL_TAB * (r - r0) : nullptr;
                const int v = tr ? tr[CT_KN] : __ldg(run_kn + r);
                const int k0 = c0 + (v & 0xFFFFFF), n = v >> 24;
                double row0[CD];
                load_row(A, k0, row0);
                const int sa = tr ? tr[CT_SA] : __ldg(run_sa + r), sb = tr ? tr[CT_SB] : __ldg(run_sb + r);
                bool remote;
                if (staged) {
                    const int s0 = rslot[2 * (r - r0)], s1 = rslot[2 * (r - r0) + 1];
                    run_pass_rec(A, rec_of(s0), rec_of(s1), I, row0, k0, n, vel, warm && p == 0, p == 0, slop);
                    remote = (s0 >= 0 && (s0 >> 20) != me) || (s1 >= 0 && (s1 >> 20) != me);
                } else {
                    run_pass(A, V, I, row0, k0, n, vel, warm && p == 0, p == 0, slop);
                    remote = true;                       // global records: other CTAs read them
                }
                int ps_[2], rs_[2], m = 0;
                const int sides[2] = {sa, sb};
#pragma unroll
                for (int sd = 0; sd < 2; sd++) {
                    const int sc = sides[sd];
                    if (sc >= 0) { ps_[m] = p; rs_[m] = sc; m++; }
                    else if (sc != LEVEL_NONE && p + 1 < P) { ps_[m] = p + 1; rs_[m] = -sc - 1; m++; }
                }
                // successor tables (their need counts and lengths), and whether any
                // successor, or any successor's other predecessor, lies in another CTA
                // (whose last arrival may then acquire these writes): then the release
                // is cluster scope
                int needs[2] = {0, 0}, lens[2] = {0, 0};
                for (int q = 0; q < m; q++) {
                    const int rs = rs_[q];
                    const int *ts = tab_of(rs);
                    needs[q] = ts ? ts[CT_NEED] : __ldg(run_need + rs);
                    lens[q] = (ts ? ts[CT_KN] : __ldg(run_kn + rs)) >> 24;
                    if (cl_home(rs, R, C) != me) remote = true;
                    else if (!ts || ts[CT_XPRED]) remote = true;
                }
                // release this entry's writes: to this CTA alone, or to the cluster
                if (remote) fence_acq_rel_cluster(); else fence_acq_rel_cta();
                for (int q = 0; q < m; q++) {
                    const int rs = rs_[q], ps = ps_[q];
                    const int h = cl_home(rs, R, C);
                    int *arr = h == me ? mine.arrived + (rs - r0)
                                       : cl_home_arrays<C>(A, cluster, csm, h, R, P, c0, smem_ints, me).arrived +
                                             (rs - cl_first(h, R, C));
                    if (atomicAdd(arr, 1) + 1 == need_of(needs[q], ps)) {
                        fence_acq_rel_cluster();         // acquire the other arrivals' writes
                        push((ps << PASS_SHIFT) | rs, rs, lens[q]);
                    }
                }
            }
        }
        __syncwarp();
    }
    if (lane == 0 && *(volatile int *)&cs.abort) atomicOr(&A.status[ST_SWEEP_TIMEOUT], 1);
    if (me == 0 && threadIdx.x == 0) A.w_levels[w] = -1;     // not tracked on the cluster sweep
    __syncthreads();
    cluster.sync();               // every entry done: records final, no CTA reaches another's memory after this
    if (staged) {
        for (int i = threadIdx.x; i < cs.n_owned; i += blockDim.x) {
            const int body = owned[i];
            const double *rec = recs + (size_t)i * CL_REC;
            for (int q = 0; q < 3; q++) {
                A.v[body * 3 + q] = rec[q];
                A.w[body * 3 + q] = rec[3 + q];
                A.pos[body * 3 + q] = rec[6 + q];
            }
        }
        if (I.s)
            for (int i = threadIdx.x; i < 3 * (k_hi - k_lo); i += blockDim.x) A.c_imp[(c0 + k_lo) * 3 + i] = I.s[i];
    }
}

// ---------------------------------------------------------------------------
// integrate positions and sleep of wide worlds (k_finalize's passes, each a
// grid launch; the union-find works on the global parent array of the world,
// roots the island's smallest index, so labels match k_finalize's):
//   phase 0: positions; per body slow / ready flags, timer, parent = self
//   phase 1: per contact: contacted flags and unions of dynamic pairs
//   phase 2: per body: island label (root)
//   phase 3: per body: a contacted body not ready marks its island not ready
//   phase 4: per body: sleep or wake, island -1 without contact, rest at zero
// ---------------------------------------------------------------------------
__global__ void k_wfinalize(Arena A, int mode, int phase) {
    if ((mode & FIN_GATED) && overflowed(A)) return;
    const int w = A.wide_w[blockIdx.y];
    if (!A.w_active[w]) return;
    const double dt = A.w_dt[w];
    const int b0 = A.w_body_off[w], nb = A.w_body_n[w], b1 = b0 + nb;
    const bool sleep = (mode & FIN_SLEEP) && (A.w_flags[w] & WF_SLEEP);
    int *flag = A.b_flag + b0, *parent = A.b_parent + b0;
    if (phase == 0) {
        for (int i = b0 + wide_tid(); i < b1; i += wide_stride()) {
            if (mode & FIN_POSITIONS) {
                const int t = A.mtype[i];
                if ((t == 2 || t == 1) && A.awake[i]) {
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
            if (!sleep) { A.b_island[i] = -1; continue; }
            const double lin2 = 0.08 * 0.08, ang2 = 0.25 * 0.25;
            const bool dyn_i = A.mtype[i] == 2;
            const bool slow = dyn_i && speed2(&A.v[i * 3]) < lin2 && speed2(&A.w[i * 3]) < ang2;
            if (slow) A.timer[i] += dt; else A.timer[i] = 0.0;
            const bool ready = slow && A.timer[i] > 0.4;
            flag[i - b0] = (slow ? BF_SLOW : 0) | (ready ? BF_READY : 0);
            parent[i - b0] = i - b0;
        }
        return;
    }
    if (!sleep) return;
    if (phase == 1) {
        if (!world_collides(A, w)) return;
        int c0, c1;
        world_contacts(A, w, c0, c1);
        for (int k = c0 + wide_tid(); k < c1; k += wide_stride()) {
            const int a = A.c_a[k], b = A.c_b[k];
            const bool da = A.mtype[a] == 2, db = A.mtype[b] == 2;
            if (da) atomicOr(&flag[a - b0], BF_CONTACTED);
            if (db) atomicOr(&flag[b - b0], BF_CONTACTED);
            if (da && db) uf_union(parent, a - b0, b - b0);
        }
    } else if (phase == 2) {
        for (int i = wide_tid(); i < nb; i += wide_stride()) A.b_island[b0 + i] = b0 + uf_find(parent, i);
    } else if (phase == 3) {
        for (int i = wide_tid(); i < nb; i += wide_stride()) {
            const int f = ((volatile int *)flag)[i];
            if ((f & BF_CONTACTED) && !(f & BF_READY)) atomicOr(&flag[A.b_island[b0 + i] - b0], BF_NOTREADY);
        }
    } else {
        for (int i = b0 + wide_tid(); i < b1; i += wide_stride()) {
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
    }
}

}  // namespace omi
