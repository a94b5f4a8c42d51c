// omi_b200: the C ABI (include/omi_b200.h) over the device arena.
//
// Host-side duties: own the device buffers and the stream, upload the scene
// tables, run the step as a CUDA graph, regrow pair/contact capacities when a
// step reports an overflow (the step is then re-run; nothing was modified),
// and copy results back for the caller. All compute is in the kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <mutex>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/omi_b200.h"
#include "capsule.cuh"
#include "wide.cuh"

using namespace omi;

namespace {

enum KernelId {
    KN_REFIT, KN_SORT, KN_PAIR_COUNT, KN_PAIR_SCAN, KN_PAIR_EMIT, KN_NARROW, KN_GJK,
    KN_CONTACT_SCAN, KN_INTEGRATE_FORCES, KN_COMPACT, KN_WAKE, KN_PREP, KN_LEVELS, KN_SOLVE,
    KN_TRIGGERS, KN_CACHE, KN_JOINTS, KN_FINALIZE, KN_COUNT
};
const char *kKernelNames[KN_COUNT] = {
    "refit", "sort", "pair_count", "pair_scan", "pair_emit", "narrow", "gjk_epa",
    "contact_scan", "integrate_forces", "contact_compact", "wake", "prep", "levels", "solve",
    "triggers", "cache_store", "joints", "integrate_positions_sleep"};

struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
};

}  // namespace

// Serving slots: per-slot capacities and the first row of each of its tables.
struct SlotTable {
    std::vector<OmiSlotCaps> caps;
    std::vector<int64_t> b0, s0, m0, p0, j0, f0, pf0;   // n + 1 prefix sums
};

struct OmiCtx {
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    std::string err;
    int64_t budget = 0;
    std::vector<Buf> statics;      // scene tables and per-body arrays
    std::vector<Buf> dyn;          // pair/contact sized buffers
    std::vector<Buf> cache;        // warm-start cache buffers (preserved on growth)
    int64_t bytes = 0;
    Arena A{};
    bool loaded = false;
    int max_world_n = 0, max_world_j = 0, sort_cap = 0, sort_block = 256;
    int level_ints = 0;            // shared ints of one k_levels block
    int sm_count = 148;            // multiprocessors of the device (persistent sweep grid)
    int fin_cap = 1;               // bodies whose sleep flags / islands k_finalize keeps in shared memory
    int stage_doubles = 0;         // doubles of world state k_iterate stages in shared memory
    int cache_cap = 0;
    bool has_triggers = false;     // some body carries a sensor shape: k_triggers runs each step
    bool has_meshes = false;       // some body is a triangle mesh: k_mesh_count / k_mesh_emit run
    int moving_meshes = 0;         // meshes (rows of the mesh tables) when one of them is kinematic, else 0
    cudaGraphExec_t graph = nullptr;
    int *h_status = nullptr;       // pinned mirror of the status words
    int64_t launches = 0;
    std::vector<float> prof_ms;
    std::vector<uint8_t> h_active;
    std::vector<int> h_body_off, h_body_n, h_joint_off;
    bool slots = false;
    SlotTable slot;                // capacities and table offsets of each slot
    // capsule-triangle host pipeline: two buffer sets, one per internal stream
    std::vector<Buf> capbufs;
    int64_t cap_chunk = 0;         // triangles one buffer set holds
    int cap_q = 0;                 // capsule rows the caps / tri_off buffers hold
    double *cap_caps = nullptr;
    int64_t *cap_off = nullptr;
    double *cap_v[2] = {}, *cap_p[2] = {}, *cap_n[2] = {}, *cap_d[2] = {};
    uint8_t *cap_h[2] = {};
    cudaStream_t cap_s[2] = {};
    cudaEvent_t cap_ev = nullptr;
    int cap_blocks = 0;            // resident k_capsule_triangles blocks per SM
    // bounds a test may lower (omi_set_limits): sweep wait polls, EPA faces, stalled run
    int spin_limit = SPIN_LIMIT_DEFAULT, epa_faces = EPA_F, stall_run = -1;
    OmiTuning tune = {8, 4, 256, 16, 128, 4, 16, 16, 32};   // launch configuration (omi_set_tuning)
    int cluster_max = 0;                        // largest thread-block cluster of k_csweep the GPU schedules
    int cluster_ints = 0;                       // shared-memory ints a k_csweep CTA may use (0: all it has)
    int joint_smem = 0;                         // doubles of shared memory a k_joints block takes
    // wide worlds (their stages on many blocks): the worlds, bodies of the largest, sort merge passes
    std::vector<int> h_wide;
    int wide_max_n = 0, wide_merge_passes = 0;
    int wide_min_bodies = 3072;                 // a colliding world with more bodies runs wide
    int64_t graph_launches = 0;                 // kernels one captured step launches
};

namespace {

int fail(OmiCtx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(OmiCtx *c, cudaError_t e, const char *where) {
    return fail(c, OMI_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e__ = (call);                             \
        if (e__ != cudaSuccess) return cuda_fail(ctx, e__, #call); \
    } while (0)

template <class T>
int alloc(OmiCtx *ctx, std::vector<Buf> &pool, T *&out, size_t n) {
    size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    bytes = (bytes + 255) & ~size_t(255);
    if (ctx->budget > 0 && ctx->bytes + (int64_t)bytes > ctx->budget)
        return fail(ctx, OMI_E_OOM, "device budget exceeded allocating " + std::to_string(bytes) + " bytes");
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    e = cudaMemsetAsync(p, 0, bytes, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemset");
    pool.push_back({p, bytes});
    ctx->bytes += (int64_t)bytes;
    out = static_cast<T *>(p);
    return 0;
}

template <class T>
int upload(OmiCtx *ctx, T *&out, const T *src, size_t n) {
    int rc = alloc(ctx, ctx->statics, out, n);
    if (rc) return rc;
    if (src && n) {
        cudaError_t e = cudaMemcpyAsync(out, src, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync H2D");
    }
    return 0;
}

void free_pool(OmiCtx *ctx, std::vector<Buf> &pool) {
    for (auto &b : pool) {
        cudaFree(b.p);
        ctx->bytes -= (int64_t)b.bytes;
    }
    pool.clear();
}

void drop_graph(OmiCtx *ctx) {
    if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
    ctx->graph = nullptr;
}

int passes_of(int flags, int iters) {
    const int p = ((flags & OMI_WF_WARM) ? 1 : 0) + std::max(iters, 0);
    return std::max(p, 1);
}

int grid_for(int n, int block, int cap) {
    int g = (n + block - 1) / block;
    return std::max(1, std::min(g, cap));
}

// shared memory (doubles) k_joints wants for one world's joints: prepared
// rows, the velocities of the joints' body range and the schedule (levels
// and order of every entry, and level starts for a chain's J + 2 iters
// levels with room to spare), capped at JOINT_SMEM_DOUBLES
int joint_smem_need(const int *ja, const int *jb, int nj, int iters) {
    if (nj <= 0) return 0;
    int lo = INT32_MAX, hi = -1;
    for (int j = 0; j < nj; j++)
        for (int b : {ja[j], jb[j]})
            if (b >= 0) { lo = std::min(lo, b); hi = std::max(hi, b); }
    const int64_t nbr = hi >= lo ? hi - lo + 1 : 0;
    const int64_t E = iters <= JOINT_WAVE_ITERS ? (int64_t)nj * std::max(iters, 0) : nj;
    const int64_t ints = nbr + 2 * E + 2 * ((int64_t)nj + 2 * std::max(iters, 0) + 66);
    const int64_t need = (int64_t)nj * JD + 6 * nbr + (ints + 1) / 2;
    return (int)std::min<int64_t>(need, JOINT_SMEM_DOUBLES);
}

// dynamic shared memory of one k_csweep CTA (what a block may hold, less its static part)
size_t sweep_cluster_smem() { return (size_t)SWEEP_SMEM_DOUBLES * sizeof(double) - 256; }

// blocks of `block` threads for n items of a wide world, at most 8 per SM
int wide_grid(const OmiCtx *ctx, int n, int block) {
    return std::max(1, std::min((n + block - 1) / block, ctx->sm_count * 8));
}

int hash_bits_for(int runs) {
    int bits = 10;
    while ((1 << bits) < 2 * runs) bits++;
    return bits;
}

// (re)allocate the pair/contact-sized buffers; the warm-start cache survives
int alloc_dynamic(OmiCtx *ctx, int pair_cap, int contact_cap) {
    drop_graph(ctx);
    cudaStreamSynchronize(ctx->stream);
    free_pool(ctx, ctx->dyn);
    Arena &A = ctx->A;
    A.pair_cap = pair_cap;
    A.contact_cap = contact_cap;
    int rc = 0;
    rc |= alloc(ctx, ctx->dyn, A.pair_a, pair_cap);
    rc |= alloc(ctx, ctx->dyn, A.pair_b, pair_cap);
    rc |= alloc(ctx, ctx->dyn, A.pair_solid, pair_cap);
    rc |= alloc(ctx, ctx->dyn, A.slot_cnt, (size_t)pair_cap + 1);
    rc |= alloc(ctx, ctx->dyn, A.slot, (size_t)pair_cap * SLOT);
    rc |= alloc(ctx, ctx->dyn, A.clip_list, pair_cap);
    rc |= alloc(ctx, ctx->dyn, A.gjk_list, pair_cap);
    rc |= alloc(ctx, ctx->dyn, A.trig_list, ctx->has_triggers ? pair_cap : 1);
    rc |= alloc(ctx, ctx->dyn, A.mesh_list, ctx->has_meshes ? pair_cap : 1);
    rc |= alloc(ctx, ctx->dyn, A.trig_out, ctx->has_triggers ? 3 * (size_t)pair_cap : 3);
    rc |= alloc(ctx, ctx->dyn, A.contact_scan, (size_t)pair_cap + 1);
    rc |= alloc(ctx, ctx->dyn, A.c_a, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.c_b, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.c_pt, (size_t)contact_cap * 3);
    rc |= alloc(ctx, ctx->dyn, A.c_n, (size_t)contact_cap * 3);
    rc |= alloc(ctx, ctx->dyn, A.c_depth, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.c_imp, (size_t)contact_cap * 3);
    rc |= alloc(ctx, ctx->dyn, A.c_data, (size_t)contact_cap * CD);
    const size_t entries = (size_t)contact_cap * A.max_passes;
    if (entries >= ((size_t)1 << 31) - 2) return fail(ctx, OMI_E_ARG, "contact capacity x sweep passes exceeds 2^31");
    rc |= alloc(ctx, ctx->dyn, A.c_order, entries);
    rc |= alloc(ctx, ctx->dyn, A.run_pa, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_pb, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_sa, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_sb, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_kn, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_need, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_done, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_tend, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.lv_scratch, 3 * (size_t)contact_cap + 2 * (size_t)A.NB + 2 * (size_t)A.W + 64);
    const bool wide = !ctx->h_wide.empty();
    rc |= alloc(ctx, ctx->dyn, A.wl_flag, wide ? contact_cap : 1);
    rc |= alloc(ctx, ctx->dyn, A.wl_scan, wide ? (size_t)contact_cap + 1 : 1);
    rc |= alloc(ctx, ctx->dyn, A.wl_list, wide ? 2 * (size_t)contact_cap + 1 : 1);
    rc |= alloc(ctx, ctx->dyn, A.run_k, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_n, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_a, contact_cap);
    rc |= alloc(ctx, ctx->dyn, A.run_b, contact_cap);
    size_t scan_n = std::max({(size_t)pair_cap, (size_t)contact_cap, (size_t)A.NB}) / SCAN_TILE + 2;
    rc |= alloc(ctx, ctx->dyn, A.scan_blocks, scan_n + 1);
    if (rc) return rc;
    // warm-start cache: up to one step's contacts plus worlds keeping old ones
    const int want_cache = 2 * contact_cap;
    if (want_cache > ctx->cache_cap) {
        std::vector<Buf> old = ctx->cache;
        Arena prev = A;
        const int prev_cap = ctx->cache_cap;
        ctx->cache.clear();
        for (int t = 0; t < 2; t++) {
            rc |= alloc(ctx, ctx->cache, A.cache_a[t], want_cache);
            rc |= alloc(ctx, ctx->cache, A.cache_b[t], want_cache);
            rc |= alloc(ctx, ctx->cache, A.cache_pt[t], (size_t)want_cache * 3);
            rc |= alloc(ctx, ctx->cache, A.cache_imp[t], (size_t)want_cache * 3);
            rc |= alloc(ctx, ctx->cache, A.hused[t], want_cache);
        }
        const int bits = hash_bits_for(want_cache);
        A.hash_mask = (1 << bits) - 1;
        for (int t = 0; t < 2; t++) {
            rc |= alloc(ctx, ctx->cache, A.hkey[t], (size_t)1 << bits);
            rc |= alloc(ctx, ctx->cache, A.hval[t], (size_t)2 << bits);
        }
        if (rc) return rc;
        for (int t = 0; t < 2; t++) {
            CK(cudaMemsetAsync(A.hkey[t], 0xff, sizeof(unsigned long long) << bits, ctx->stream));
            if (prev_cap > 0) {
                CK(cudaMemcpyAsync(A.cache_a[t], prev.cache_a[t], sizeof(int) * prev_cap, cudaMemcpyDeviceToDevice, ctx->stream));
                CK(cudaMemcpyAsync(A.cache_b[t], prev.cache_b[t], sizeof(int) * prev_cap, cudaMemcpyDeviceToDevice, ctx->stream));
                CK(cudaMemcpyAsync(A.cache_pt[t], prev.cache_pt[t], sizeof(double) * 3 * prev_cap, cudaMemcpyDeviceToDevice, ctx->stream));
                CK(cudaMemcpyAsync(A.cache_imp[t], prev.cache_imp[t], sizeof(double) * 3 * prev_cap, cudaMemcpyDeviceToDevice, ctx->stream));
            }
        }
        CK(cudaMemsetAsync(A.hused_n, 0, sizeof(int) * 4, ctx->stream));
        ctx->cache_cap = want_cache;
        cudaStreamSynchronize(ctx->stream);
        for (auto &b : old) { cudaFree(b.p); ctx->bytes -= (int64_t)b.bytes; }
        for (int t = 0; t < 2; t++) {
            k_hash_rebuild<<<std::max(1, A.W), 128, 0, ctx->stream>>>(A, t);
            ctx->launches++;
        }
        CK(cudaGetLastError());
    }
    return 0;
}

void launch_scan(OmiCtx *ctx, const int *in, int *out, int n_const, const int *n_ptr, int cap,
                 const int *gate_scan, int gate_idx, int gate_cap) {
    const int tiles = std::max(1, (cap + SCAN_TILE - 1) / SCAN_TILE);
    k_scan_tiles<<<tiles, 1024, 0, ctx->stream>>>(in, out, n_const, n_ptr, gate_scan, gate_idx, gate_cap, ctx->A.scan_blocks);
    k_scan_top<<<1, 1024, 0, ctx->stream>>>(ctx->A.scan_blocks, tiles, gate_scan, gate_idx, gate_cap);
    k_scan_add<<<tiles, 1024, 0, ctx->stream>>>(out, n_const, n_ptr, ctx->A.scan_blocks, tiles, gate_scan, gate_idx, gate_cap);
    ctx->launches += 3;
}

constexpr int SM_CAP = 148 * 16;

// the kernels of each stage; `prof` records an event after each stage
struct Prof {
    cudaEvent_t ev[KN_COUNT + 1];
    bool on = false;
};

void mark(OmiCtx *ctx, Prof *pf, int k) {
    if (pf && pf->on) cudaEventRecord(pf->ev[k + 1], ctx->stream);
}

void stage_refit(OmiCtx *ctx, Prof *pf) {
    Arena &A = ctx->A;
    k_refit<<<grid_for(A.NB, 256, SM_CAP), 256, 0, ctx->stream>>>(A);
    ctx->launches++;
    mark(ctx, pf, KN_REFIT);
}

void stage_broadphase(OmiCtx *ctx, Prof *pf) {
    Arena &A = ctx->A;
    const size_t smem = (size_t)ctx->sort_cap * (2 * sizeof(double) + 2 * sizeof(int));
    k_sort<true><<<std::min(A.W, 65535), ctx->sort_block, smem, ctx->stream>>>(A, ctx->sort_cap);
    ctx->launches++;
    if (A.n_wide) {
        const int tiles = (ctx->wide_max_n + WSORT_TILE - 1) / WSORT_TILE;
        k_wsort_tiles<<<dim3(tiles, A.n_wide), WSORT_THREADS, (size_t)WSORT_TILE * 24, ctx->stream>>>(A);
        int src = 0;
        for (int j = 0, width = WSORT_TILE; j < ctx->wide_merge_passes; j++, width *= 2, src ^= 1)
            k_wsort_merge<<<dim3(wide_grid(ctx, ctx->wide_max_n, 256), A.n_wide), 256, 0, ctx->stream>>>(A, width, src);
        k_wsort_rows<<<dim3(wide_grid(ctx, ctx->wide_max_n, 256), A.n_wide), 256, 0, ctx->stream>>>(A, src);
        ctx->launches += 2 + ctx->wide_merge_passes;
    }
    mark(ctx, pf, KN_SORT);
    const OmiTuning &t = ctx->tune;
    const int pgrid = grid_for(A.NB * 32, t.pair_block, ctx->sm_count * t.pair_blocks_per_sm);
    k_pair_count<<<pgrid, t.pair_block, 0, ctx->stream>>>(A);
    ctx->launches++;
    mark(ctx, pf, KN_PAIR_COUNT);
    launch_scan(ctx, A.pair_cnt, A.pair_scan, A.NB, nullptr, A.NB, nullptr, 0, 0);
    k_pair_check<<<1, 1, 0, ctx->stream>>>(A);
    ctx->launches++;
    mark(ctx, pf, KN_PAIR_SCAN);
    k_pair_emit<<<pgrid, t.pair_block, 0, ctx->stream>>>(A);
    ctx->launches++;
    mark(ctx, pf, KN_PAIR_EMIT);
}

void stage_narrow(OmiCtx *ctx, Prof *pf) {
    Arena &A = ctx->A;
    if (ctx->moving_meshes) {
        k_mesh_refresh<<<std::min(ctx->moving_meshes, 148), MESH_REFRESH_THREADS, 0, ctx->stream>>>(A, ctx->moving_meshes);
        ctx->launches++;
    }
    const int nb = ctx->tune.narrow_block, gw = ctx->tune.gjk_warps;
    k_narrow<<<grid_for(A.pair_cap, nb, SM_CAP), nb, 0, ctx->stream>>>(A);
    k_edge_clip<<<grid_for(A.pair_cap, nb, SM_CAP), nb, 0, ctx->stream>>>(A);
    ctx->launches += 2;
    mark(ctx, pf, KN_NARROW);
    k_gjk<<<ctx->sm_count * (16 / gw), 32 * gw, gw * sizeof(EpaWork), ctx->stream>>>(A);
    ctx->launches++;
    if (ctx->has_meshes) {
        k_mesh_count<<<148 * 4, 128, 4 * sizeof(EpaWork), ctx->stream>>>(A);
        ctx->launches++;
    }
    mark(ctx, pf, KN_GJK);
    launch_scan(ctx, A.slot_cnt, A.contact_scan, 0, A.pair_scan + A.NB, A.pair_cap, A.pair_scan, A.NB, A.pair_cap);
    k_contact_check<<<1, 1, 0, ctx->stream>>>(A);
    ctx->launches++;
    mark(ctx, pf, KN_CONTACT_SCAN);
}

void stage_compact(OmiCtx *ctx, Prof *pf) {
    Arena &A = ctx->A;
    k_contact_compact<<<grid_for(A.pair_cap, 128, SM_CAP), 128, 0, ctx->stream>>>(A);
    ctx->launches++;
    if (ctx->has_meshes) {
        k_mesh_emit<<<148 * 4, 128, 4 * sizeof(EpaWork), ctx->stream>>>(A);
        ctx->launches++;
    }
    mark(ctx, pf, KN_COMPACT);
}

void stage_solve(OmiCtx *ctx, Prof *pf) {
    Arena &A = ctx->A;
    const int nw = A.n_wide;
    const int cgrid = wide_grid(ctx, A.contact_cap, 256);     // contacts of wide worlds
    if (nw) cudaMemsetAsync(A.wide_state, 0, sizeof(int) * WIDE_STATE_INTS * nw, ctx->stream);
    k_wake<<<std::min(A.W, 65535), WAKE_THREADS, 0, ctx->stream>>>(A);
    if (nw) {
        k_wwake<<<dim3(cgrid, nw), 256, 0, ctx->stream>>>(A, 0);
        k_wwake<<<dim3(cgrid, nw), 256, 0, ctx->stream>>>(A, 1);
        ctx->launches += 2;
    }
    mark(ctx, pf, KN_WAKE);
    k_prep<<<grid_for(A.contact_cap, PREP_THREADS, SM_CAP), PREP_THREADS, (size_t)PREP_THREADS * CD * sizeof(double), ctx->stream>>>(A);
    mark(ctx, pf, KN_PREP);
    k_levels<<<std::min(A.W, 65535), LEVEL_THREADS, (size_t)ctx->level_ints * sizeof(int), ctx->stream>>>(A, ctx->level_ints);
    if (nw) {
        const int kgrid = wide_grid(ctx, A.contact_cap, 256);
        k_wl_flags<<<kgrid, 256, 0, ctx->stream>>>(A);
        launch_scan(ctx, A.wl_flag, A.wl_scan, 0, A.k_total, A.contact_cap, A.pair_scan, A.NB, A.pair_cap);
        k_wl_runs<<<kgrid, 256, 0, ctx->stream>>>(A);
        k_wl_count<<<dim3(cgrid, nw), 256, 0, ctx->stream>>>(A);
        launch_scan(ctx, A.wl_cnt, A.wl_bstart, A.NB, nullptr, A.NB, nullptr, 0, 0);
        k_wl_fill<<<dim3(cgrid, nw), 256, 0, ctx->stream>>>(A);
        k_wl_links<<<dim3(cgrid, nw), 256, 0, ctx->stream>>>(A);
        ctx->launches += 5;
    }
    mark(ctx, pf, KN_LEVELS);
    const size_t sweep_smem = (size_t)ctx->stage_doubles * sizeof(double);
    if (ctx->tune.sweep_warps == 4)
        k_iterate<4><<<std::min(A.W, ctx->sm_count), 128, sweep_smem, ctx->stream>>>(A, ctx->stage_doubles,
                                                                                     ctx->tune.sweep_max_split);
    else
        k_iterate<8><<<std::min(A.W, ctx->sm_count), 256, sweep_smem, ctx->stream>>>(A, ctx->stage_doubles,
                                                                                     ctx->tune.sweep_max_split);
    ctx->launches += 4;
    const int csmem_full = (int)(sweep_cluster_smem() / sizeof(int));
    const int csmem_ints = ctx->cluster_ints > 0 ? std::min(ctx->cluster_ints, csmem_full) : csmem_full;
    const int wb = std::min(ctx->tune.wide_sweep_blocks, ctx->sm_count);
    if (nw && (ctx->tune.wide_cluster == 16 || ctx->tune.wide_cluster == 8)) {
        // the cluster sweeps a world whose records fit its shared memory; the
        // many-block sweep after it takes the world otherwise (it returns at
        // once when the cluster swept); with one wide block chosen the
        // cluster sweeps every world itself
        const int handoff = wb > 1;
        for (int wi = 0; wi < nw; wi++) {
            if (ctx->tune.wide_cluster == 16)
                k_csweep<16><<<16, SWEEP_THREADS, sweep_cluster_smem(), ctx->stream>>>(A, wi, csmem_ints, handoff);
            else
                k_csweep<8><<<8, SWEEP_THREADS, sweep_cluster_smem(), ctx->stream>>>(A, wi, csmem_ints, handoff);
            ctx->launches++;
            if (handoff) {
                k_wsweep_init<<<cgrid, 256, 0, ctx->stream>>>(A, wi);
                k_wsweep_seed<<<cgrid, 256, 0, ctx->stream>>>(A, wi);
                k_wsweep<<<wb, SWEEP_THREADS, 0, ctx->stream>>>(A, wi);
                ctx->launches += 3;
            }
        }
    } else if (nw && ctx->tune.wide_sweep_blocks == 1) {
        // one block per wide world: the per-world sweep with its shared-memory staging
        k_wsweep_one<<<nw, SWEEP_THREADS, sweep_smem, ctx->stream>>>(A, ctx->stage_doubles);
        ctx->launches++;
    } else {
        for (int wi = 0; wi < nw; wi++) {      // one wide world at a time, on wb SMs
            k_wsweep_init<<<cgrid, 256, 0, ctx->stream>>>(A, wi);
            k_wsweep_seed<<<cgrid, 256, 0, ctx->stream>>>(A, wi);
            k_wsweep<<<wb, SWEEP_THREADS, 0, ctx->stream>>>(A, wi);
            ctx->launches += 3;
        }
    }
    mark(ctx, pf, KN_SOLVE);
    if (ctx->has_triggers) {
        k_triggers<<<148 * 4, 128, 4 * sizeof(EpaWork), ctx->stream>>>(A);
        ctx->launches++;
    }
    mark(ctx, pf, KN_TRIGGERS);
    k_cache_plan<<<1, 1024, 0, ctx->stream>>>(A);
    k_hash_clear<<<grid_for(ctx->cache_cap, 256, SM_CAP), 256, 0, ctx->stream>>>(A);
    // every world's entries (wide ones included) over the whole grid
    const int kgrid_cache = grid_for(ctx->cache_cap, 256, SM_CAP);
    k_cache_copy<<<kgrid_cache, 256, 0, ctx->stream>>>(A);
    k_hash_build<<<kgrid_cache, 256, 0, ctx->stream>>>(A);
    k_flip<<<1, 1, 0, ctx->stream>>>(A);
    ctx->launches += 5;
    mark(ctx, pf, KN_CACHE);
}

void stage_joints(OmiCtx *ctx, Prof *pf, int gated) {
    Arena &A = ctx->A;
    if (A.NJ > 0) {
        const int jsd = std::max(ctx->joint_smem, 256);
        k_joints<<<std::min(A.W, 65535), 32, (size_t)jsd * sizeof(double), ctx->stream>>>(A, gated, jsd);
        ctx->launches++;
    }
    mark(ctx, pf, KN_JOINTS);
}

// integrate positions and / or sleep (k_finalize's modes) for every world:
// one block per world, and the wide worlds' grid passes
void stage_finalize(OmiCtx *ctx, int mode) {
    Arena &A = ctx->A;
    k_finalize<<<std::min(A.W, 65535), 256, (size_t)2 * ctx->fin_cap * sizeof(int), ctx->stream>>>(A, mode, ctx->fin_cap);
    ctx->launches++;
    if (A.n_wide) {
        const int bgrid = wide_grid(ctx, ctx->wide_max_n, 256), cgrid = wide_grid(ctx, A.contact_cap, 256);
        k_wfinalize<<<dim3(bgrid, A.n_wide), 256, 0, ctx->stream>>>(A, mode, 0);
        ctx->launches++;
        if (mode & FIN_SLEEP) {
            k_wfinalize<<<dim3(cgrid, A.n_wide), 256, 0, ctx->stream>>>(A, mode, 1);
            for (int ph = 2; ph <= 4; ph++) k_wfinalize<<<dim3(bgrid, A.n_wide), 256, 0, ctx->stream>>>(A, mode, ph);
            ctx->launches += 4;
        }
    }
}

// one full step (world.py:410-430) for every active world
void enqueue_step(OmiCtx *ctx, Prof *pf) {
    Arena &A = ctx->A;
    if (pf && pf->on) cudaEventRecord(pf->ev[0], ctx->stream);
    stage_refit(ctx, pf);
    stage_broadphase(ctx, pf);
    stage_narrow(ctx, pf);
    k_integrate_forces<<<grid_for(A.NB, 256, SM_CAP), 256, 0, ctx->stream>>>(A, 1);
    ctx->launches++;
    mark(ctx, pf, KN_INTEGRATE_FORCES);
    stage_compact(ctx, pf);
    stage_solve(ctx, pf);
    stage_joints(ctx, pf, 1);
    stage_finalize(ctx, FIN_POSITIONS | FIN_SLEEP | FIN_COUNT | FIN_GATED);
    mark(ctx, pf, KN_FINALIZE);
}

int reset_status(OmiCtx *ctx) {
    return cudaMemsetAsync(ctx->A.status, 0, sizeof(int) * ST_WORDS, ctx->stream) == cudaSuccess ? 0 : -1;
}

int read_status(OmiCtx *ctx) {
    cudaError_t e = cudaMemcpyAsync(ctx->h_status, ctx->A.status, sizeof(int) * ST_WORDS,
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "status D2H");
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
    return 0;
}

// grow after an overflow recorded in the status words
int grow_for_overflow(OmiCtx *ctx) {
    int *st = ctx->h_status;
    int pair_cap = ctx->A.pair_cap, contact_cap = ctx->A.contact_cap;
    if (st[ST_OVERFLOW] == 1) {
        const int need = st[ST_PAIRS_NEEDED];
        pair_cap = std::max(pair_cap * 2, need + need / 2 + 1024);
        contact_cap = std::max(contact_cap, 2 * pair_cap);
    } else if (st[ST_OVERFLOW] == 2) {
        const int need = st[ST_CONTACTS_NEEDED];
        contact_cap = std::max(contact_cap * 2, need + need / 2 + 1024);
    }
    return alloc_dynamic(ctx, pair_cap, contact_cap);
}

int capture(OmiCtx *ctx) {
    drop_graph(ctx);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamBeginCapture");
    const int64_t before = ctx->launches;
    enqueue_step(ctx, nullptr);
    e = cudaStreamEndCapture(ctx->stream, &g);
    ctx->graph_launches = ctx->launches - before;
    ctx->launches = before;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&ctx->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
    return 0;
}

int64_t step_launches(OmiCtx *ctx) {
    return ctx->graph_launches;        // kernels of the captured step (counted while capturing)
}

// errors the status words of completed steps carry: a sweep wait that ran
// out (the step did not complete), or pairs whose EPA polytope outgrew its
// bound (the step completed, but those pairs' contacts were dropped where the
// reference's unbounded EPA would have made one)
int status_errors(OmiCtx *ctx) {
    const int *st = ctx->h_status;
    if (st[ST_BOUNDS]) {
        static const char *sites[] = {"?", "narrowphase pair body", "shape or hull point range",
                                      "contact body", "solver row body outside its world",
                                      "sweep successor run", "joint body outside its world",
                                      "contact body outside its world (islands)", "filter-matrix row"};
        const int site = st[ST_BOUNDS_SITE];
        return fail(ctx, OMI_E_BOUNDS, std::to_string(st[ST_BOUNDS]) + " device index check(s) failed, the first at " +
                                           sites[site >= 1 && site <= 8 ? site : 0] + " (index " +
                                           std::to_string(st[ST_BOUNDS_INDEX]) +
                                           "); the accesses were skipped and the step's results are not valid");
    }
    if (st[ST_SWEEP_TIMEOUT])
        return fail(ctx, OMI_E_TIMEOUT, "contact sweep wait timed out (the step did not complete; "
                                        "restore the worlds' state before stepping on)");
    if (st[ST_EPA_LIMIT])
        return fail(ctx, OMI_E_LIMIT, std::to_string(st[ST_EPA_LIMIT]) +
                                          " convex pair test(s) outgrew the bounded EPA polytope; their "
                                          "contacts were dropped (the step completed)");
    return 0;
}

int run_steps(OmiCtx *ctx, int n, bool sync) {
    if (!ctx->loaded) return fail(ctx, OMI_E_STATE, "omi_step before omi_load");
    int remaining = n;
    int guard = 0;
    while (remaining > 0) {
        if (reset_status(ctx)) return fail(ctx, OMI_E_CUDA, "status reset");
        if (!ctx->graph) {
            int rc = capture(ctx);
            if (rc) return rc;
        }
        for (int s = 0; s < remaining; s++) {
            cudaError_t e = cudaGraphLaunch(ctx->graph, ctx->stream);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphLaunch");
            ctx->launches += step_launches(ctx);
        }
        if (!sync) return 0;
        int rc = read_status(ctx);
        if (rc) return rc;
        if (ctx->h_status[ST_SWEEP_TIMEOUT] || ctx->h_status[ST_BOUNDS]) return status_errors(ctx);
        const int done = ctx->h_status[ST_STEPS_DONE];
        remaining -= done;
        if (remaining > 0) {
            if (!ctx->h_status[ST_OVERFLOW] || ++guard > 16)
                return fail(ctx, OMI_E_STATE, "step did not complete (no overflow recorded)");
            rc = grow_for_overflow(ctx);
            if (rc) return rc;
        }
    }
    return status_errors(ctx);
}

template <class T>
int put(OmiCtx *ctx, T *dst, const T *src, size_t n) {
    if (!n) return 0;
    cudaError_t e = cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "slot upload");
}

int check_world(OmiCtx *ctx, int w) {
    if (!ctx->loaded) return fail(ctx, OMI_E_STATE, "no scene loaded");
    if (w < 0 || w >= ctx->A.W) return fail(ctx, OMI_E_ARG, "world index out of range");
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int omi_create(int device, OmiCtx **out) {
    if (!out) return OMI_E_ARG;
    *out = nullptr;
    OmiCtx *ctx = new OmiCtx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { int rc = cuda_fail(ctx, e, "cudaSetDevice"); *out = ctx; return rc; }
    e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) { int rc = cuda_fail(ctx, e, "cudaStreamCreate"); *out = ctx; return rc; }
    ctx->stream = ctx->own;
    e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) { int rc = cuda_fail(ctx, e, "cudaDeviceGetAttribute"); *out = ctx; return rc; }
    e = cudaMallocHost(&ctx->h_status, sizeof(int) * ST_WORDS);
    if (e != cudaSuccess) { int rc = cuda_fail(ctx, e, "cudaMallocHost"); *out = ctx; return rc; }
    const struct { const void *fn; int bytes; const char *name; } smem[] = {
        {(const void *)k_gjk, 8 * (int)sizeof(EpaWork), "k_gjk"},
        {(const void *)k_triggers, 4 * (int)sizeof(EpaWork), "k_triggers"},
        {(const void *)k_mesh_count, 4 * (int)sizeof(EpaWork), "k_mesh_count"},
        {(const void *)k_mesh_emit, 4 * (int)sizeof(EpaWork), "k_mesh_emit"},
        {(const void *)k_sort<true>, 8192 * 24, "k_sort"},
        {(const void *)k_iterate<8>, SWEEP_SMEM_DOUBLES * (int)sizeof(double), "k_iterate<8>"},
        {(const void *)k_iterate<4>, SWEEP_SMEM_DOUBLES * (int)sizeof(double), "k_iterate<4>"},
        {(const void *)k_levels, LEVEL_SMEM_INTS * (int)sizeof(int), "k_levels"},
        {(const void *)k_finalize, 2 * 8192 * (int)sizeof(int), "k_finalize"},
        {(const void *)k_prep, PREP_THREADS * CD * (int)sizeof(double), "k_prep"},
        {(const void *)k_wsort_tiles, WSORT_TILE * 24, "k_wsort_tiles"},
        {(const void *)k_wsweep_one, SWEEP_SMEM_DOUBLES * (int)sizeof(double), "k_wsweep_one"},
        {(const void *)k_joints, JOINT_SMEM_DOUBLES * (int)sizeof(double), "k_joints"},
    };
    for (const auto &f : smem) {
        e = cudaFuncSetAttribute(f.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, f.bytes);
        if (e != cudaSuccess) {
            int rc = cuda_fail(ctx, e, (std::string("cudaFuncSetAttribute ") + f.name).c_str());
            *out = ctx;
            return rc;
        }
    }
    // the cluster sweep: 16 CTAs when the GPU schedules such clusters, else 8
    ctx->cluster_max = 0;
    {
        const int bytes = (int)sweep_cluster_smem();
        if (cudaFuncSetAttribute(k_csweep<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess &&
            cudaFuncSetAttribute(k_csweep<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess &&
            cudaFuncSetAttribute(k_csweep<16>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
            for (int c : {16, 8}) {
                cudaLaunchConfig_t cfg = {};
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = c; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
                cfg.gridDim = dim3(c); cfg.blockDim = dim3(SWEEP_THREADS); cfg.dynamicSmemBytes = bytes;
                cfg.attrs = at; cfg.numAttrs = 1;
                int n = 0;
                const cudaError_t q = c == 16 ? cudaOccupancyMaxActiveClusters(&n, (void *)k_csweep<16>, &cfg)
                                              : cudaOccupancyMaxActiveClusters(&n, (void *)k_csweep<8>, &cfg);
                if (q == cudaSuccess && n >= 1) { ctx->cluster_max = c; break; }
                cudaGetLastError();
            }
        }
        cudaGetLastError();
        ctx->tune.wide_cluster = ctx->cluster_max;
    }
    *out = ctx;
    return 0;
}

int omi_destroy(OmiCtx *ctx) {
    if (!ctx) return 0;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_graph(ctx);
    free_pool(ctx, ctx->dyn);
    free_pool(ctx, ctx->cache);
    free_pool(ctx, ctx->statics);
    for (int k = 0; k < 2; k++)
        if (ctx->cap_s[k]) { cudaStreamSynchronize(ctx->cap_s[k]); cudaStreamDestroy(ctx->cap_s[k]); }
    if (ctx->cap_ev) cudaEventDestroy(ctx->cap_ev);
    free_pool(ctx, ctx->capbufs);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return 0;
}

const char *omi_last_error(OmiCtx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int omi_set_stream(OmiCtx *ctx, void *stream) {
    if (!ctx) return OMI_E_ARG;
    cudaStreamSynchronize(ctx->stream);
    drop_graph(ctx);
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own;
    return 0;
}

int omi_set_budget(OmiCtx *ctx, int64_t bytes) {
    if (!ctx) return OMI_E_ARG;
    ctx->budget = bytes;
    return 0;
}

int64_t omi_device_bytes(OmiCtx *ctx) { return ctx ? ctx->bytes : 0; }
int64_t omi_launch_count(OmiCtx *ctx) { return ctx ? ctx->launches : 0; }
const char *omi_kernel_name(int32_t i) { return (i >= 0 && i < KN_COUNT) ? kKernelNames[i] : ""; }

// Host-side check of a whole-arena scene and the per-body tables derived from
// it (refit kind and half extents, sensor and AABB shapes, mesh rows). Every
// index a kernel follows is range-checked here, so no kernel reads out of
// bounds; nothing touches the device.
struct SceneDerived {
    std::vector<int> body_world, tshape, rshape, vol_off, body_mesh;
    std::vector<int8_t> kind;
    std::vector<double> half;
    bool sensors = false;
    int max_n = 0, max_nc = 0, max_j = 0, n_meshes = 0, n_tris = 0;
};

#define BAD(code, msg) do { err = (msg); return (code); } while (0)

static int derive_scene(const OmiScene *s, SceneDerived &D, std::string &err) {
    if (!s) BAD(OMI_E_ARG, "null scene");
    const int W = s->n_worlds, NB = s->n_bodies;
    if (W <= 0 || NB < 0 || !s->w_body_off || !s->w_joint_off || s->w_body_off[0] != 0 || s->w_body_off[W] != NB)
        BAD(OMI_E_ARG, "inconsistent world/body offsets");
    if (s->n_shapes < 0 || s->n_materials < 0 || s->n_points < 0 || s->n_joints < 0 || s->n_pair_friction < 0 ||
        s->n_filter_bytes < 0 || s->n_volumes < 0 || s->n_meshes < 0)
        BAD(OMI_E_ARG, "negative table size");
    for (int w = 0; w < W; w++) {
        if (s->w_body_off[w + 1] < s->w_body_off[w]) BAD(OMI_E_ARG, "world offsets decrease");
        if (s->w_joint_off[w + 1] < s->w_joint_off[w]) BAD(OMI_E_ARG, "joint offsets decrease");
        const int rows = s->w_filter_rows[w];
        if (rows < 1 || rows > 4096 || s->w_filter_off[w] < 0 ||
            (int64_t)s->w_filter_off[w] + (int64_t)rows * rows > s->n_filter_bytes)
            BAD(OMI_E_ARG, "filter matrix range out of bounds");
        if (s->w_pf_off[w] < 0 || s->w_pf_n[w] < 0 || s->w_pf_off[w] + s->w_pf_n[w] > s->n_pair_friction)
            BAD(OMI_E_ARG, "pair-friction range out of bounds");
        if (s->w_iters[w] < 0 || s->w_joint_iters[w] < 0) BAD(OMI_E_ARG, "negative iteration count");
    }
    if (s->w_joint_off[0] != 0 || s->w_joint_off[W] != s->n_joints) BAD(OMI_E_ARG, "inconsistent joint offsets");
    D = SceneDerived{};
    D.body_world.assign(NB, 0);
    D.kind.assign(NB, 0);
    D.half.assign((size_t)NB * 3, 0.0);
    D.tshape.assign(NB, -1);
    D.rshape.assign(NB, -1);
    if (s->trigger_shape)
        for (int i = 0; i < NB; i++) {
            const int t = s->trigger_shape[i];
            if (t < -1 || t >= s->n_shapes) BAD(OMI_E_ARG, "trigger shape index out of range");
            D.tshape[i] = t;
            D.sensors |= t >= 0;
        }
    D.vol_off.assign(W + 1, 0);
    if (s->w_vol_off) {
        for (int w = 0; w <= W; w++) D.vol_off[w] = s->w_vol_off[w];
        if (D.vol_off[0] != 0 || D.vol_off[W] != s->n_volumes) BAD(OMI_E_ARG, "inconsistent volume offsets");
        for (int w = 0; w < W; w++)
            if (D.vol_off[w + 1] < D.vol_off[w]) BAD(OMI_E_ARG, "volume offsets decrease");
    } else if (s->n_volumes != 0) {
        BAD(OMI_E_ARG, "gravity volumes without w_vol_off");
    }
    for (int w = 0; w < W; w++) {
        const int n = s->w_body_off[w + 1] - s->w_body_off[w];
        D.max_n = std::max(D.max_n, n);
        if (s->w_flags[w] & OMI_WF_COLLISION) D.max_nc = std::max(D.max_nc, n);
        for (int i = s->w_body_off[w]; i < s->w_body_off[w + 1]; i++) {
            D.body_world[i] = w;
            if (s->filter_row[i] < 0 || s->filter_row[i] >= s->w_filter_rows[w])
                BAD(OMI_E_ARG, "filter row out of range");
        }
    }
    for (int i = 0; i < NB; i++) {
        if (s->shape[i] >= s->n_shapes || s->shape[i] < -1) BAD(OMI_E_ARG, "shape index out of range");
        // the AABB comes from the collider, else the sensor (world.py:452-455)
        const int sh = s->shape[i] >= 0 ? s->shape[i] : D.tshape[i];
        D.rshape[i] = sh;
        if (s->motion_type[i] < 0 || s->motion_type[i] > 2) BAD(OMI_E_ARG, "motion type");
        if (s->material[i] >= s->n_materials || s->material[i] < -1) BAD(OMI_E_ARG, "material index out of range");
        if (sh < 0) continue;
        const int t = s->shape_type[sh];
        double *half = D.half.data();
        if (t == OMI_SHAPE_SPHERE) {
            D.kind[i] = 1;
            for (int c = 0; c < 3; c++) half[i * 3 + c] = s->shape_radius[sh];
        } else if (t == OMI_SHAPE_BOX) {
            D.kind[i] = 2;
            for (int c = 0; c < 3; c++) half[i * 3 + c] = 0.5 * s->shape_size[sh * 3 + c];
        } else if (t == OMI_SHAPE_CONVEX) {
            D.kind[i] = 3;
            if (s->shape_pt_cnt[sh] < 1 || s->shape_pt_off[sh] < 0 ||
                s->shape_pt_off[sh] + s->shape_pt_cnt[sh] > s->n_points)
                BAD(OMI_E_ARG, "convex point range out of bounds");
        } else if (t == OMI_SHAPE_CAPSULE) {
            D.kind[i] = 4;
            half[i * 3] = s->shape_radius[sh];
            half[i * 3 + 1] = 0.5 * s->shape_size[sh * 3 + 1];
            half[i * 3 + 2] = 0.0;
        } else if (t == OMI_SHAPE_TRIMESH) {
            D.kind[i] = 5;
            if (s->shape_pt_cnt[sh] < 1 || s->shape_pt_off[sh] < 0 ||
                s->shape_pt_off[sh] + s->shape_pt_cnt[sh] > s->n_points)
                BAD(OMI_E_ARG, "mesh point range out of bounds");
            if (s->shape[i] != sh || s->motion_type[i] == 2)
                BAD(OMI_E_UNSUPPORTED, "triangle meshes are taken as static or kinematic colliders only");
        } else {
            BAD(OMI_E_UNSUPPORTED, "shape type not supported on the device path");
        }
    }
    // triangle meshes: every mesh body listed once, its tables in range
    D.body_mesh.assign(NB, -1);
    const int NMESH = s->mesh_body ? s->n_meshes : 0;
    D.n_meshes = NMESH;
    if (NMESH) {
        if (!s->mesh_tri_off || !s->mesh_grid_i) BAD(OMI_E_ARG, "mesh tables missing");
        if (s->mesh_tri_off[0] != 0) BAD(OMI_E_ARG, "mesh triangle offsets must start at 0");
        for (int m = 0; m < NMESH; m++) {
            const int b = s->mesh_body[m];
            if (b < 0 || b >= NB || D.kind[b] != 5 || D.body_mesh[b] >= 0) BAD(OMI_E_ARG, "mesh body");
            if (s->mesh_tri_off[m + 1] < s->mesh_tri_off[m]) BAD(OMI_E_ARG, "mesh triangle offsets decrease");
            const int *gi = &s->mesh_grid_i[m * 4];
            if (!gi[0] && (gi[1] < 1 || gi[2] < 1 || gi[3] < 1)) BAD(OMI_E_ARG, "mesh grid shape");
            D.body_mesh[b] = m;
        }
        D.n_tris = s->mesh_tri_off[NMESH];
        if (!s->tri_idx) BAD(OMI_E_ARG, "mesh tables without tri_idx");
        for (int m = 0; m < NMESH; m++) {
            const int b = s->mesh_body[m], sh = s->shape[b];
            for (int t = s->mesh_tri_off[m]; t < s->mesh_tri_off[m + 1]; t++)
                for (int j = 0; j < 3; j++)
                    if (s->tri_idx[t * 3 + j] < 0 || s->tri_idx[t * 3 + j] >= s->shape_pt_cnt[sh])
                        BAD(OMI_E_ARG, "mesh triangle vertex index out of range");
        }
    }
    for (int i = 0; i < NB; i++)
        if (D.kind[i] == 5 && D.body_mesh[i] < 0) BAD(OMI_E_ARG, "a mesh body without its triangle tables");
    for (int p = 0; p < s->n_pair_friction; p++)
        if (s->pf_a[p] >= s->n_materials || s->pf_b[p] >= s->n_materials)
            BAD(OMI_E_ARG, "pair-friction material out of range");
    for (int w = 0; w < W; w++) {
        for (int j = s->w_joint_off[w]; j < s->w_joint_off[w + 1]; j++) {
            if (s->j_type[j] < 0 || s->j_type[j] > 2) BAD(OMI_E_ARG, "joint type");
            if (s->j_a[j] >= NB || s->j_b[j] >= NB || s->j_a[j] < -1 || s->j_b[j] < -1)
                BAD(OMI_E_ARG, "joint body out of range");
            if (s->j_type[j] == OMI_JOINT_MOTOR && s->j_a[j] < 0) BAD(OMI_E_ARG, "motor without a body");
            // a joint's bodies belong to its own world (each world's joints are solved by one block)
            if ((s->j_a[j] >= 0 && D.body_world[s->j_a[j]] != w) || (s->j_b[j] >= 0 && D.body_world[s->j_b[j]] != w))
                BAD(OMI_E_ARG, "joint body outside the joint's world");
        }
        D.max_j = std::max(D.max_j, s->w_joint_off[w + 1] - s->w_joint_off[w]);
    }
    return 0;
}
#undef BAD

static int load_impl(OmiCtx *ctx, const OmiScene *s, const int *body_n, const int *joint_n) {
    if (!ctx || !s) return OMI_E_ARG;
    // check everything before the previous arena is released: a refused scene leaves it loaded
    SceneDerived D;
    {
        std::string msg;
        const int vrc = derive_scene(s, D, msg);
        if (vrc) return fail(ctx, vrc, msg);
    }
    CK(cudaSetDevice(ctx->device));
    cudaStreamSynchronize(ctx->stream);
    drop_graph(ctx);
    free_pool(ctx, ctx->dyn);
    free_pool(ctx, ctx->cache);
    free_pool(ctx, ctx->statics);
    ctx->cache_cap = 0;
    ctx->loaded = false;
    const int W = s->n_worlds, NB = s->n_bodies;
    const std::vector<int> &body_world = D.body_world, &tshape = D.tshape, &rshape = D.rshape;
    const std::vector<int> &vol_off = D.vol_off, &body_mesh = D.body_mesh;
    const std::vector<int8_t> &kind = D.kind;
    const std::vector<double> &half = D.half;
    const bool sensors = D.sensors;
    const int max_n = D.max_n, max_nc = D.max_nc, max_j = D.max_j, NMESH = D.n_meshes, n_tris = D.n_tris;
    Arena &A = ctx->A;
    A = Arena{};
    A.W = W; A.NB = NB; A.NS = s->n_shapes; A.NM = s->n_materials; A.NJ = s->n_joints;
    A.NPTS = s->n_points;
    A.spin_limit = ctx->spin_limit;
    A.epa_faces = ctx->epa_faces;
    A.stall_run = ctx->stall_run;
    A.sweep_claim = ctx->tune.sweep_claim;
    int rc = 0;
    // worlds
    rc |= upload(ctx, const_cast<int *&>(A.w_body_off), s->w_body_off, W + 1);
    rc |= upload(ctx, const_cast<int *&>(A.w_body_n), body_n, W);
    rc |= upload(ctx, const_cast<int *&>(A.w_joint_n), joint_n, W);
    ctx->h_body_off.assign(s->w_body_off, s->w_body_off + W + 1);
    ctx->h_body_n.assign(body_n, body_n + W);
    ctx->h_joint_off.assign(s->w_joint_off, s->w_joint_off + W + 1);
    {
        std::vector<int> sched(W);
        for (int w = 0; w < W; w++) sched[w] = w;
        std::stable_sort(sched.begin(), sched.end(), [&](int x, int y) { return body_n[x] > body_n[y]; });
        rc |= upload(ctx, const_cast<int *&>(A.w_sched), sched.data(), W);
    }
    rc |= upload(ctx, const_cast<double *&>(A.w_g), s->w_gravity, (size_t)W * 3);
    rc |= upload(ctx, const_cast<double *&>(A.w_dt), s->w_dt, W);
    rc |= upload(ctx, const_cast<int *&>(A.w_iters), s->w_iters, W);
    rc |= upload(ctx, const_cast<int *&>(A.w_jiters), s->w_joint_iters, W);
    rc |= upload(ctx, const_cast<int *&>(A.w_flags), s->w_flags, W);
    ctx->h_active.assign(W, 1);
    for (int w = 0; w < W; w++) ctx->h_active[w] = (s->w_flags[w] & OMI_WF_ACTIVE) ? 1 : 0;
    rc |= upload(ctx, const_cast<uint8_t *&>(A.w_active), ctx->h_active.data(), W);
    rc |= upload(ctx, const_cast<double *&>(A.w_def_damp), s->w_default_damp, (size_t)W * 2);
    rc |= upload(ctx, const_cast<double *&>(A.w_solver), s->w_solver, (size_t)W * 2);
    rc |= upload(ctx, const_cast<int *&>(A.w_filter_off), s->w_filter_off, W);
    rc |= upload(ctx, const_cast<int *&>(A.w_filter_rows), s->w_filter_rows, W);
    rc |= upload(ctx, const_cast<int *&>(A.w_pf_off), s->w_pf_off, W);
    rc |= upload(ctx, const_cast<int *&>(A.w_pf_n), s->w_pf_n, W);
    rc |= upload(ctx, const_cast<int *&>(A.w_joint_off), s->w_joint_off, W + 1);
    // bodies
    rc |= upload(ctx, A.pos, s->pos, (size_t)NB * 3);
    rc |= upload(ctx, A.q, s->q, (size_t)NB * 4);
    rc |= upload(ctx, A.v, s->v, (size_t)NB * 3);
    rc |= upload(ctx, A.w, s->w, (size_t)NB * 3);
    rc |= upload(ctx, A.prev_pos, s->pos, (size_t)NB * 3);
    rc |= upload(ctx, A.prev_q, s->q, (size_t)NB * 4);
    rc |= upload(ctx, const_cast<double *&>(A.inv_mass), s->inv_mass, NB);
    rc |= upload(ctx, const_cast<double *&>(A.inv_inertia), s->inv_inertia, (size_t)NB * 3);
    rc |= upload(ctx, const_cast<double *&>(A.gf), s->gravity_factor, NB);
    rc |= upload(ctx, const_cast<double *&>(A.ld), s->lin_damp, NB);
    rc |= upload(ctx, const_cast<double *&>(A.ad), s->ang_damp, NB);
    rc |= upload(ctx, const_cast<double *&>(A.qd), s->quad_drag, NB);
    rc |= upload(ctx, A.timer, s->sleep_timer, NB);
    rc |= upload(ctx, A.awake, s->awake, NB);
    rc |= upload(ctx, const_cast<int *&>(A.mtype), s->motion_type, NB);
    rc |= upload(ctx, const_cast<int *&>(A.shape), s->shape, NB);
    rc |= upload(ctx, const_cast<int *&>(A.material), s->material, NB);
    rc |= upload(ctx, const_cast<int *&>(A.material_key), s->material_key, NB);
    rc |= upload(ctx, const_cast<int *&>(A.filter_row), s->filter_row, NB);
    rc |= upload(ctx, const_cast<int *&>(A.body_world), body_world.data(), NB);
    rc |= upload(ctx, const_cast<int8_t *&>(A.kind), kind.data(), NB);
    rc |= upload(ctx, const_cast<double *&>(A.half), half.data(), (size_t)NB * 3);
    rc |= upload(ctx, const_cast<int *&>(A.tshape), tshape.data(), NB);
    rc |= upload(ctx, const_cast<int *&>(A.body_mesh), body_mesh.data(), NB);
    rc |= upload(ctx, const_cast<int *&>(A.mesh_tri_off), NMESH ? s->mesh_tri_off : nullptr, (size_t)NMESH + 1);
    rc |= upload(ctx, const_cast<int *&>(A.mesh_grid_i), NMESH ? s->mesh_grid_i : nullptr, (size_t)NMESH * 4);
    rc |= upload(ctx, const_cast<double *&>(A.mesh_grid_d), NMESH ? s->mesh_grid_d : nullptr, (size_t)NMESH * 7);
    rc |= upload(ctx, const_cast<double *&>(A.tri_verts), n_tris ? s->tri_verts : nullptr, (size_t)n_tris * 9);
    rc |= upload(ctx, const_cast<double *&>(A.tri_box), n_tris ? s->tri_box : nullptr, (size_t)n_tris * 6);
    rc |= upload(ctx, const_cast<int *&>(A.tri_cells), n_tris ? s->tri_cells : nullptr, (size_t)n_tris * 6);
    rc |= upload(ctx, const_cast<uint8_t *&>(A.tri_big), n_tris ? s->tri_big : nullptr, n_tris);
    rc |= upload(ctx, const_cast<int *&>(A.tri_idx), n_tris ? s->tri_idx : nullptr, (size_t)n_tris * 3);
    rc |= upload(ctx, const_cast<int *&>(A.mesh_body_of), NMESH ? s->mesh_body : nullptr, NMESH);
    ctx->has_meshes = NMESH > 0;
    ctx->moving_meshes = 0;
    for (int m = 0; m < NMESH; m++)
        if (s->motion_type[s->mesh_body[m]] != 0) ctx->moving_meshes = NMESH;
    rc |= upload(ctx, const_cast<int *&>(A.rshape), rshape.data(), NB);
    ctx->has_triggers = sensors;
    // gravity volumes
    const int NV = s->w_vol_off ? s->n_volumes : 0;
    rc |= upload(ctx, const_cast<int *&>(A.w_vol_off), vol_off.data(), W + 1);
    rc |= upload(ctx, const_cast<int *&>(A.vol_kind), NV ? s->vol_kind : nullptr, NV);
    rc |= upload(ctx, const_cast<double *&>(A.vol_g), NV ? s->vol_g : nullptr, NV);
    rc |= upload(ctx, const_cast<double *&>(A.vol_field), NV ? s->vol_field : nullptr, (size_t)NV * 3);
    rc |= upload(ctx, const_cast<double *&>(A.vol_rc), NV ? s->vol_rc : nullptr, (size_t)NV * 3);
    rc |= upload(ctx, const_cast<double *&>(A.vol_rr), NV ? s->vol_rr : nullptr, (size_t)NV * 3);
    rc |= alloc(ctx, ctx->statics, A.aabb_min, (size_t)NB * 3);
    rc |= alloc(ctx, ctx->statics, A.aabb_max, (size_t)NB * 3);
    rc |= alloc(ctx, ctx->statics, A.invIw, (size_t)NB * 9);
    // shapes, materials, filters
    rc |= upload(ctx, const_cast<int *&>(A.shape_type), s->shape_type, s->n_shapes);
    rc |= upload(ctx, const_cast<double *&>(A.shape_radius), s->shape_radius, s->n_shapes);
    rc |= upload(ctx, const_cast<double *&>(A.shape_size), s->shape_size, (size_t)s->n_shapes * 3);
    rc |= upload(ctx, const_cast<int *&>(A.pt_off), s->shape_pt_off, s->n_shapes);
    rc |= upload(ctx, const_cast<int *&>(A.pt_cnt), s->shape_pt_cnt, s->n_shapes);
    rc |= upload(ctx, const_cast<double *&>(A.points), s->points, (size_t)s->n_points * 3);
    rc |= upload(ctx, const_cast<double *&>(A.mat_dynf), s->mat_dynf, s->n_materials);
    rc |= upload(ctx, const_cast<double *&>(A.mat_rest), s->mat_rest, s->n_materials);
    rc |= upload(ctx, const_cast<int *&>(A.mat_fcomb), s->mat_fcomb, s->n_materials);
    rc |= upload(ctx, const_cast<int *&>(A.mat_rcomb), s->mat_rcomb, s->n_materials);
    rc |= upload(ctx, const_cast<int *&>(A.pf_a), s->pf_a, s->n_pair_friction);
    rc |= upload(ctx, const_cast<int *&>(A.pf_b), s->pf_b, s->n_pair_friction);
    rc |= upload(ctx, const_cast<double *&>(A.pf_mu), s->pf_mu, s->n_pair_friction);
    rc |= upload(ctx, const_cast<uint8_t *&>(A.filter_matrix), s->filter_matrix, s->n_filter_bytes);
    // joints
    const int NJ = s->n_joints;
    rc |= upload(ctx, const_cast<int *&>(A.j_type), s->j_type, NJ);
    rc |= upload(ctx, const_cast<int *&>(A.j_a), s->j_a, NJ);
    rc |= upload(ctx, const_cast<int *&>(A.j_b), s->j_b, NJ);
    rc |= upload(ctx, const_cast<double *&>(A.j_anchor), s->j_anchor, (size_t)NJ * 3);
    rc |= upload(ctx, const_cast<double *&>(A.j_anchor_b), s->j_anchor_b, (size_t)NJ * 3);
    rc |= upload(ctx, const_cast<double *&>(A.j_axis), s->j_axis, (size_t)NJ * 3);
    rc |= upload(ctx, const_cast<double *&>(A.j_target), s->j_target, NJ);
    rc |= upload(ctx, const_cast<double *&>(A.j_max_force), s->j_max_force, NJ);
    rc |= upload(ctx, A.j_local_a, s->j_local_a, (size_t)NJ * 3);
    rc |= upload(ctx, A.j_local_b, s->j_local_b, (size_t)NJ * 3);
    rc |= upload(ctx, A.j_length, s->j_length, NJ);
    rc |= upload(ctx, A.j_accum, s->j_accum, NJ);
    rc |= upload(ctx, A.j_has_local_a, s->j_has_local_a, NJ);
    rc |= upload(ctx, A.j_has_local_b, s->j_has_local_b, NJ);
    rc |= upload(ctx, A.j_has_length, s->j_has_length, NJ);
    rc |= alloc(ctx, ctx->statics, A.j_data, (size_t)NJ * JD);
    rc |= alloc(ctx, ctx->statics, A.j_level, (size_t)NJ * JOINT_WAVE_ITERS);
    rc |= alloc(ctx, ctx->statics, A.j_order, (size_t)NJ * JOINT_WAVE_ITERS);
    rc |= alloc(ctx, ctx->statics, A.j_level_start, 2 * ((size_t)NJ * JOINT_WAVE_ITERS + W + 1));
    // per-body scratch
    rc |= alloc(ctx, ctx->statics, A.order, NB);
    rc |= alloc(ctx, ctx->statics, A.sorted_x, NB);
    rc |= alloc(ctx, ctx->statics, A.srt_box, (size_t)NB * 8);
    rc |= alloc(ctx, ctx->statics, A.srt_info, NB);
    rc |= alloc(ctx, ctx->statics, A.pair_end, NB);
    rc |= alloc(ctx, ctx->statics, A.pair_mask, NB);
    for (int t = 0; t < 2; t++) {
        rc |= alloc(ctx, ctx->statics, A.sort_k[t], NB);
        rc |= alloc(ctx, ctx->statics, A.sort_v[t], NB);
    }
    rc |= alloc(ctx, ctx->statics, A.pair_cnt, NB);
    rc |= alloc(ctx, ctx->statics, A.pair_scan, (size_t)NB + 1);
    rc |= alloc(ctx, ctx->statics, A.b_last, NB);
    rc |= alloc(ctx, ctx->statics, A.b_parent, NB);
    rc |= alloc(ctx, ctx->statics, A.b_island, NB);
    rc |= alloc(ctx, ctx->statics, A.b_flag, NB);
    rc |= alloc(ctx, ctx->statics, A.w_levels, W);
    rc |= alloc(ctx, ctx->statics, A.w_runs, W);
    rc |= alloc(ctx, ctx->statics, A.gjk_n, 1);
    rc |= alloc(ctx, ctx->statics, A.trig_n, 1);
    rc |= alloc(ctx, ctx->statics, A.mesh_n, 1);
    rc |= alloc(ctx, ctx->statics, A.clip_n, 1);
    rc |= alloc(ctx, ctx->statics, A.sweep_next, 1);
    for (int t = 0; t < 2; t++) {
        rc |= alloc(ctx, ctx->statics, A.w_cache_off[t], W);
        rc |= alloc(ctx, ctx->statics, A.w_cache_n[t], W);
    }
    rc |= alloc(ctx, ctx->statics, A.w_cache_new, W + 1);
    rc |= alloc(ctx, ctx->statics, A.hused_n, 4);
    rc |= alloc(ctx, ctx->statics, A.parity, 1);
    rc |= alloc(ctx, ctx->statics, A.status, ST_WORDS);
    // wide worlds: colliding worlds above wide_min_bodies run their per-world stages on many blocks
    {
        ctx->h_wide.clear();
        std::vector<uint8_t> flag(W, 0);
        ctx->wide_max_n = 0;
        for (int w = 0; w < W; w++) {
            const int n = s->w_body_off[w + 1] - s->w_body_off[w];
            if ((s->w_flags[w] & OMI_WF_COLLISION) && n > ctx->wide_min_bodies) {
                flag[w] = 1;
                ctx->h_wide.push_back(w);
                ctx->wide_max_n = std::max(ctx->wide_max_n, n);
            }
        }
        A.n_wide = (int)ctx->h_wide.size();
        ctx->wide_merge_passes = 0;
        for (int64_t t = WSORT_TILE; t < ctx->wide_max_n; t *= 2) ctx->wide_merge_passes++;
        rc |= upload(ctx, const_cast<int *&>(A.wide_w), ctx->h_wide.empty() ? nullptr : ctx->h_wide.data(),
                     std::max<size_t>(ctx->h_wide.size(), 1));
        rc |= upload(ctx, const_cast<uint8_t *&>(A.w_wide), flag.data(), W);
        rc |= alloc(ctx, ctx->statics, A.wide_state, (size_t)std::max(A.n_wide, 1) * WIDE_STATE_INTS);
        rc |= alloc(ctx, ctx->statics, A.wl_cnt, A.n_wide ? (size_t)NB : 1);
        rc |= alloc(ctx, ctx->statics, A.wl_bstart, A.n_wide ? (size_t)NB + 1 : 1);
        rc |= alloc(ctx, ctx->statics, A.k_total, 1);
    }
    if (rc) return rc;
    ctx->max_world_n = max_n;
    ctx->max_world_j = max_j;
    int max_nc_narrow = 0;          // the largest colliding world the one-block-per-world sort takes
    for (int w = 0; w < W; w++) {
        const int n = s->w_body_off[w + 1] - s->w_body_off[w];
        if ((s->w_flags[w] & OMI_WF_COLLISION) && n <= ctx->wide_min_bodies) max_nc_narrow = std::max(max_nc_narrow, n);
    }
    ctx->sort_cap = std::min(std::max(max_nc_narrow, 1), 8192);
    ctx->sort_block = max_nc_narrow > 2048 ? 1024 : (max_nc_narrow > 512 ? 512 : 256);
    // sleep flags and union-find parents of the largest world (two ints per body, <= 64 KB)
    ctx->fin_cap = std::min(std::max(max_n, 1), 8192);
    // body buckets of the largest world: 2 ints per body + 2 per run (~1.5 runs per body)
    ctx->level_ints = (int)std::min<int64_t>(LEVEL_SMEM_INTS, 8 * (int64_t)std::max(max_nc, 1) + 1024);
    A.max_passes = 1;
    for (int w = 0; w < W; w++) A.max_passes = std::max(A.max_passes, passes_of(s->w_flags[w], s->w_iters[w]));
    // the largest world's per-run tables (4 ints, ~1.5 runs per body),
    // velocities (6 per body), impulses (~2 contacts per body, 3 each) and work
    // ring (~1.5 runs per body x passes)
    ctx->stage_doubles = (int)std::min<int64_t>(SWEEP_SMEM_DOUBLES,
                                                (int64_t)std::max(max_nc, 1) * (16 + A.max_passes) + 64);
    ctx->joint_smem = 0;
    for (int w = 0; w < W; w++) {
        const int j0 = s->w_joint_off[w], nj = s->w_joint_off[w + 1] - j0;
        if (nj > 0)
            ctx->joint_smem = std::max(ctx->joint_smem,
                                       joint_smem_need(s->j_a + j0, s->j_b + j0, nj, s->w_joint_iters[w]));
    }
    const int pair_cap = std::max(4096, 4 * NB);
    rc = alloc_dynamic(ctx, pair_cap, 2 * pair_cap);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->loaded = true;
    return 0;
}

int omi_load(OmiCtx *ctx, const OmiScene *s) {
    if (!ctx || !s || s->n_worlds <= 0) return OMI_E_ARG;
    std::vector<int> bn(s->n_worlds), jn(s->n_worlds);
    for (int w = 0; w < s->n_worlds; w++) {
        bn[w] = s->w_body_off[w + 1] - s->w_body_off[w];
        jn[w] = s->w_joint_off[w + 1] - s->w_joint_off[w];
    }
    ctx->slots = false;
    return load_impl(ctx, s, bn.data(), jn.data());
}

int omi_reserve_slots_each(OmiCtx *ctx, int32_t n, const OmiSlotCaps *caps) {
    if (!ctx || !caps || n <= 0) return fail(ctx, OMI_E_ARG, "bad slot capacities");
    for (int w = 0; w < n; w++) {
        const OmiSlotCaps &c = caps[w];
        if (c.bodies <= 0 || c.filter_rows < 1 || c.shapes < 0 || c.materials < 0 || c.points < 0 ||
            c.joints < 0 || c.pair_friction < 0 || c.bodies > (1 << 24) || c.filter_rows > 4096)
            return fail(ctx, OMI_E_ARG, "bad slot capacities");
    }
    // per-slot table offsets: prefix sums of the capacities (empty tables keep one row)
    SlotTable t;
    t.caps.assign(caps, caps + n);
    for (auto *v : {&t.b0, &t.s0, &t.m0, &t.p0, &t.j0, &t.f0, &t.pf0}) v->assign(n + 1, 0);
    for (int w = 0; w < n; w++) {
        const OmiSlotCaps &c = caps[w];
        t.b0[w + 1] = t.b0[w] + c.bodies;
        t.s0[w + 1] = t.s0[w] + std::max(c.shapes, 1);
        t.m0[w + 1] = t.m0[w] + std::max(c.materials, 1);
        t.p0[w + 1] = t.p0[w] + std::max(c.points, 1);
        t.j0[w + 1] = t.j0[w] + c.joints;
        t.f0[w + 1] = t.f0[w] + (int64_t)c.filter_rows * c.filter_rows;
        t.pf0[w + 1] = t.pf0[w] + c.pair_friction;
    }
    if (t.b0[n] > (1 << 30) || t.f0[n] > (1 << 30) || t.s0[n] > (1 << 30) || t.p0[n] > (1 << 30) ||
        t.j0[n] > (1 << 30) || t.m0[n] > (1 << 30) || t.pf0[n] > (1 << 30))
        return fail(ctx, OMI_E_ARG, "slot arena too large");
    const size_t NB = t.b0[n], NS = t.s0[n], NM = t.m0[n], NP = t.p0[n], NJ = t.j0[n], NF = t.f0[n], NPF = t.pf0[n];
    std::vector<int> body_off(n + 1), joint_off(n + 1), zeros_w(n, 0), frows(n, 1), foff(n), pfoff(n), iters(n, 10);
    for (int w = 0; w <= n; w++) { body_off[w] = (int)t.b0[w]; joint_off[w] = (int)t.j0[w]; }
    for (int w = 0; w < n; w++) { foff[w] = (int)t.f0[w]; pfoff[w] = (int)t.pf0[w]; }
    std::vector<double> g(3 * n, 0.0), dt(n, 1.0 / 60.0), damp(2 * n, 0.0), solver(2 * n);
    for (int w = 0; w < n; w++) { solver[2 * w] = 0.5; solver[2 * w + 1] = 0.005; }
    std::vector<double> zb(NB * 4, 0.0), qb(NB * 4, 0.0);
    for (size_t i = 0; i < NB; i++) qb[i * 4 + 3] = 1.0;
    std::vector<int> zi(std::max(NB, NS), 0), neg(std::max(NB, NJ) + 1, -1);
    std::vector<uint8_t> ones(NB, 1), fm(NF, 1), zu(std::max(NJ, (size_t)1), 0);
    std::vector<double> zs(std::max({NS, NM, NP, NJ, NPF}) * 3 + 3, 0.0);
    std::vector<int> zsi(std::max({NS, NM, NJ, NPF}) + 1, 0);
    OmiScene s{};
    s.n_worlds = n;
    s.w_body_off = body_off.data(); s.w_gravity = g.data(); s.w_dt = dt.data();
    s.w_iters = iters.data(); s.w_joint_iters = iters.data(); s.w_flags = zeros_w.data();
    s.w_default_damp = damp.data(); s.w_solver = solver.data();
    s.w_filter_off = foff.data(); s.w_filter_rows = frows.data();
    s.w_pf_off = pfoff.data(); s.w_pf_n = zeros_w.data(); s.w_joint_off = joint_off.data();
    s.n_bodies = (int)NB;
    s.pos = zb.data(); s.q = qb.data(); s.v = zb.data(); s.w = zb.data();
    s.inv_mass = zb.data(); s.inv_inertia = zb.data(); s.gravity_factor = zb.data();
    s.lin_damp = zb.data(); s.ang_damp = zb.data(); s.quad_drag = zb.data(); s.sleep_timer = zb.data();
    s.motion_type = zi.data(); s.shape = neg.data(); s.material = neg.data(); s.material_key = neg.data();
    s.filter_row = zi.data(); s.awake = ones.data();
    s.n_shapes = (int)NS; s.shape_type = zsi.data(); s.shape_radius = zs.data(); s.shape_size = zs.data();
    s.shape_pt_off = zsi.data(); s.shape_pt_cnt = zsi.data(); s.n_points = (int)NP; s.points = zs.data();
    s.n_materials = (int)NM; s.mat_dynf = zs.data(); s.mat_rest = zs.data(); s.mat_fcomb = zsi.data(); s.mat_rcomb = zsi.data();
    s.n_pair_friction = (int)NPF; s.pf_a = zsi.data(); s.pf_b = zsi.data(); s.pf_mu = zs.data();
    s.n_filter_bytes = (int)NF; s.filter_matrix = fm.data();
    s.n_joints = (int)NJ; s.j_type = zsi.data(); s.j_a = neg.data(); s.j_b = neg.data();
    s.j_anchor = zs.data(); s.j_anchor_b = zs.data(); s.j_local_a = zs.data(); s.j_local_b = zs.data();
    s.j_has_local_a = zu.data(); s.j_has_local_b = zu.data(); s.j_length = zs.data(); s.j_has_length = zu.data();
    s.j_axis = zs.data(); s.j_target = zs.data(); s.j_max_force = zs.data(); s.j_accum = zs.data();
    // empty slots: no live bodies, no joints, inactive
    int rc = load_impl(ctx, &s, zeros_w.data(), zeros_w.data());
    if (rc) return rc;
    ctx->slots = true;
    ctx->slot = std::move(t);
    return 0;
}

int omi_reserve_slots(OmiCtx *ctx, int32_t n, const OmiSlotCaps *caps) {
    if (!ctx || !caps || n <= 0) return fail(ctx, OMI_E_ARG, "bad slot capacities");
    std::vector<OmiSlotCaps> each(n, *caps);
    return omi_reserve_slots_each(ctx, n, each.data());
}

int omi_load_world(OmiCtx *ctx, int32_t slot, const OmiScene *o) {
    if (!ctx || !o) return OMI_E_ARG;
    if (!ctx->loaded || !ctx->slots) return fail(ctx, OMI_E_STATE, "omi_reserve_slots first");
    Arena &A = ctx->A;
    if (slot < 0 || slot >= A.W) return fail(ctx, OMI_E_ARG, "slot out of range");
    const SlotTable &T = ctx->slot;
    const OmiSlotCaps &c = T.caps[slot];
    if (o->n_worlds != 1) return fail(ctx, OMI_E_ARG, "one world per slot");
    const int n = o->n_bodies, ns = o->n_shapes, nm = o->n_materials, np_ = o->n_points;
    const int nj = o->n_joints, rows = o->w_filter_rows[0], npf = o->n_pair_friction;
    if (n > c.bodies || ns > c.shapes || nm > c.materials || np_ > c.points || nj > c.joints ||
        rows > c.filter_rows || rows < 1 || npf > c.pair_friction || o->n_filter_bytes < rows * rows)
        return fail(ctx, OMI_E_ARG, "world exceeds the slot capacities");
    {
        const int need = passes_of(o->w_flags[0], o->w_iters[0]);
        if (need > A.max_passes) {
            A.max_passes = need;
            const int rc0 = alloc_dynamic(ctx, A.pair_cap, A.contact_cap);
            if (rc0) return rc0;
        }
    }
    const int b0 = (int)T.b0[slot], s0 = (int)T.s0[slot], m0 = (int)T.m0[slot];
    const int p0 = (int)T.p0[slot], j0 = (int)T.j0[slot];
    std::vector<int> shape(n), mat(n), body_world(n, slot);
    std::vector<int8_t> kind(n, 0);
    std::vector<double> half((size_t)n * 3, 0.0);
    for (int i = 0; i < n; i++) {
        const int sh = o->shape[i];
        if (o->motion_type[i] < 0 || o->motion_type[i] > 2) return fail(ctx, OMI_E_ARG, "motion type");
        if (o->filter_row[i] < 0 || o->filter_row[i] >= rows) return fail(ctx, OMI_E_ARG, "filter row");
        if (o->material[i] >= nm || o->material[i] < -1) return fail(ctx, OMI_E_ARG, "material index");
        mat[i] = o->material[i] < 0 ? -1 : o->material[i] + m0;
        shape[i] = sh < 0 ? -1 : sh + s0;
        if (sh < 0) continue;
        if (sh >= ns) return fail(ctx, OMI_E_ARG, "shape index");
        const int t = o->shape_type[sh];
        if (t == OMI_SHAPE_SPHERE) { kind[i] = 1; for (int k = 0; k < 3; k++) half[i * 3 + k] = o->shape_radius[sh]; }
        else if (t == OMI_SHAPE_BOX) { kind[i] = 2; for (int k = 0; k < 3; k++) half[i * 3 + k] = 0.5 * o->shape_size[sh * 3 + k]; }
        else if (t == OMI_SHAPE_CAPSULE) {
            kind[i] = 4;
            half[i * 3] = o->shape_radius[sh]; half[i * 3 + 1] = 0.5 * o->shape_size[sh * 3 + 1]; half[i * 3 + 2] = 0.0;
        }
        else if (t == OMI_SHAPE_TRIMESH) return fail(ctx, OMI_E_UNSUPPORTED, "serving slots do not take triangle meshes");
        else if (t == OMI_SHAPE_CONVEX) {
            kind[i] = 3;
            if (o->shape_pt_cnt[sh] < 1 || o->shape_pt_off[sh] < 0 || o->shape_pt_off[sh] + o->shape_pt_cnt[sh] > np_)
                return fail(ctx, OMI_E_ARG, "convex point range");
        } else return fail(ctx, OMI_E_UNSUPPORTED, "shape type not supported on the device path");
    }
    if ((o->w_vol_off && o->n_volumes > 0))
        return fail(ctx, OMI_E_UNSUPPORTED, "serving slots do not take gravity volumes");
    if (o->trigger_shape)
        for (int i = 0; i < n; i++)
            if (o->trigger_shape[i] >= 0) return fail(ctx, OMI_E_UNSUPPORTED, "serving slots do not take sensors");
    std::vector<int> ptoff(ns);
    for (int k = 0; k < ns; k++) ptoff[k] = o->shape_pt_off[k] + p0;
    std::vector<int> ja(nj), jb(nj);
    for (int j = 0; j < nj; j++) {
        if (o->j_type[j] < 0 || o->j_type[j] > 2) return fail(ctx, OMI_E_ARG, "joint type");
        if (o->j_a[j] >= n || o->j_b[j] >= n) return fail(ctx, OMI_E_ARG, "joint body");
        if (o->j_type[j] == OMI_JOINT_MOTOR && o->j_a[j] < 0) return fail(ctx, OMI_E_ARG, "motor body");
        ja[j] = o->j_a[j] < 0 ? -1 : o->j_a[j] + b0;
        jb[j] = o->j_b[j] < 0 ? -1 : o->j_b[j] + b0;
    }
    {   // a world whose joints want more of k_joints' shared memory re-captures the step
        const int need = joint_smem_need(o->j_a, o->j_b, nj, o->w_joint_iters[0]);
        if (need > ctx->joint_smem) {
            cudaStreamSynchronize(ctx->stream);
            drop_graph(ctx);
            ctx->joint_smem = need;
        }
    }
    int rc = 0;
    rc |= put(ctx, A.pos + (size_t)b0 * 3, o->pos, (size_t)n * 3);
    rc |= put(ctx, A.q + (size_t)b0 * 4, o->q, (size_t)n * 4);
    rc |= put(ctx, A.prev_pos + (size_t)b0 * 3, o->pos, (size_t)n * 3);
    rc |= put(ctx, A.prev_q + (size_t)b0 * 4, o->q, (size_t)n * 4);
    rc |= put(ctx, A.v + (size_t)b0 * 3, o->v, (size_t)n * 3);
    rc |= put(ctx, A.w + (size_t)b0 * 3, o->w, (size_t)n * 3);
    rc |= put(ctx, const_cast<double *>(A.inv_mass) + b0, o->inv_mass, n);
    rc |= put(ctx, const_cast<double *>(A.inv_inertia) + (size_t)b0 * 3, o->inv_inertia, (size_t)n * 3);
    rc |= put(ctx, const_cast<double *>(A.gf) + b0, o->gravity_factor, n);
    rc |= put(ctx, const_cast<double *>(A.ld) + b0, o->lin_damp, n);
    rc |= put(ctx, const_cast<double *>(A.ad) + b0, o->ang_damp, n);
    rc |= put(ctx, const_cast<double *>(A.qd) + b0, o->quad_drag, n);
    rc |= put(ctx, A.timer + b0, o->sleep_timer, n);
    rc |= put(ctx, A.awake + b0, o->awake, n);
    rc |= put(ctx, const_cast<int *>(A.mtype) + b0, o->motion_type, n);
    rc |= put(ctx, const_cast<int *>(A.shape) + b0, shape.data(), n);
    rc |= put(ctx, const_cast<int *>(A.rshape) + b0, shape.data(), n);
    rc |= put(ctx, const_cast<int *>(A.material) + b0, mat.data(), n);
    rc |= put(ctx, const_cast<int *>(A.material_key) + b0, o->material_key, n);
    rc |= put(ctx, const_cast<int *>(A.filter_row) + b0, o->filter_row, n);
    rc |= put(ctx, const_cast<int8_t *>(A.kind) + b0, kind.data(), n);
    rc |= put(ctx, const_cast<double *>(A.half) + (size_t)b0 * 3, half.data(), (size_t)n * 3);
    rc |= put(ctx, const_cast<int *>(A.shape_type) + s0, o->shape_type, ns);
    rc |= put(ctx, const_cast<double *>(A.shape_radius) + s0, o->shape_radius, ns);
    rc |= put(ctx, const_cast<double *>(A.shape_size) + (size_t)s0 * 3, o->shape_size, (size_t)ns * 3);
    rc |= put(ctx, const_cast<int *>(A.pt_off) + s0, ptoff.data(), ns);
    rc |= put(ctx, const_cast<int *>(A.pt_cnt) + s0, o->shape_pt_cnt, ns);
    rc |= put(ctx, const_cast<double *>(A.points) + (size_t)p0 * 3, o->points, (size_t)np_ * 3);
    rc |= put(ctx, const_cast<double *>(A.mat_dynf) + m0, o->mat_dynf, nm);
    rc |= put(ctx, const_cast<double *>(A.mat_rest) + m0, o->mat_rest, nm);
    rc |= put(ctx, const_cast<int *>(A.mat_fcomb) + m0, o->mat_fcomb, nm);
    rc |= put(ctx, const_cast<int *>(A.mat_rcomb) + m0, o->mat_rcomb, nm);
    const int pf0 = (int)T.pf0[slot], f0 = (int)T.f0[slot];
    rc |= put(ctx, const_cast<int *>(A.pf_a) + pf0, o->pf_a, npf);
    rc |= put(ctx, const_cast<int *>(A.pf_b) + pf0, o->pf_b, npf);
    rc |= put(ctx, const_cast<double *>(A.pf_mu) + pf0, o->pf_mu, npf);
    rc |= put(ctx, const_cast<uint8_t *>(A.filter_matrix) + f0, o->filter_matrix, (size_t)rows * rows);
    rc |= put(ctx, const_cast<int *>(A.j_type) + j0, o->j_type, nj);
    rc |= put(ctx, const_cast<int *>(A.j_a) + j0, ja.data(), nj);
    rc |= put(ctx, const_cast<int *>(A.j_b) + j0, jb.data(), nj);
    rc |= put(ctx, const_cast<double *>(A.j_anchor) + (size_t)j0 * 3, o->j_anchor, (size_t)nj * 3);
    rc |= put(ctx, const_cast<double *>(A.j_anchor_b) + (size_t)j0 * 3, o->j_anchor_b, (size_t)nj * 3);
    rc |= put(ctx, const_cast<double *>(A.j_axis) + (size_t)j0 * 3, o->j_axis, (size_t)nj * 3);
    rc |= put(ctx, const_cast<double *>(A.j_target) + j0, o->j_target, nj);
    rc |= put(ctx, const_cast<double *>(A.j_max_force) + j0, o->j_max_force, nj);
    rc |= put(ctx, A.j_local_a + (size_t)j0 * 3, o->j_local_a, (size_t)nj * 3);
    rc |= put(ctx, A.j_local_b + (size_t)j0 * 3, o->j_local_b, (size_t)nj * 3);
    rc |= put(ctx, A.j_length + j0, o->j_length, nj);
    rc |= put(ctx, A.j_accum + j0, o->j_accum, nj);
    rc |= put(ctx, A.j_has_local_a + j0, o->j_has_local_a, nj);
    rc |= put(ctx, A.j_has_local_b + j0, o->j_has_local_b, nj);
    rc |= put(ctx, A.j_has_length + j0, o->j_has_length, nj);
    rc |= put(ctx, const_cast<double *>(A.w_g) + (size_t)slot * 3, o->w_gravity, 3);
    rc |= put(ctx, const_cast<double *>(A.w_dt) + slot, o->w_dt, 1);
    rc |= put(ctx, const_cast<int *>(A.w_iters) + slot, o->w_iters, 1);
    rc |= put(ctx, const_cast<int *>(A.w_jiters) + slot, o->w_joint_iters, 1);
    rc |= put(ctx, const_cast<int *>(A.w_flags) + slot, o->w_flags, 1);
    rc |= put(ctx, const_cast<double *>(A.w_def_damp) + (size_t)slot * 2, o->w_default_damp, 2);
    rc |= put(ctx, const_cast<double *>(A.w_solver) + (size_t)slot * 2, o->w_solver, 2);
    rc |= put(ctx, const_cast<int *>(A.w_filter_rows) + slot, &rows, 1);
    rc |= put(ctx, const_cast<int *>(A.w_pf_n) + slot, &npf, 1);
    rc |= put(ctx, const_cast<int *>(A.w_body_n) + slot, &n, 1);
    rc |= put(ctx, const_cast<int *>(A.w_joint_n) + slot, &nj, 1);
    const int zero2[2] = {0, 0};
    for (int t = 0; t < 2; t++) rc |= put(ctx, A.w_cache_n[t] + slot, zero2, 1);
    if (rc) return rc;
    ctx->h_body_n[slot] = n;
    {
        std::vector<int> sched(A.W);
        for (int w = 0; w < A.W; w++) sched[w] = w;
        std::stable_sort(sched.begin(), sched.end(),
                         [&](int x, int y) { return ctx->h_body_n[x] > ctx->h_body_n[y]; });
        rc |= put(ctx, const_cast<int *>(A.w_sched), sched.data(), A.W);
        CK(cudaStreamSynchronize(ctx->stream));
    }
    ctx->h_active[slot] = (o->w_flags[0] & OMI_WF_ACTIVE) ? 1 : 0;
    rc = put(ctx, const_cast<uint8_t *>(A.w_active) + slot, &ctx->h_active[slot], 1);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_world_rows(OmiCtx *ctx, int32_t w, int32_t *first, int32_t *count) {
    int rc = check_world(ctx, w);
    if (rc) return rc;
    if (first) *first = ctx->h_body_off[w];
    if (count) *count = ctx->h_body_n[w];
    return 0;
}

int omi_set_world_params(OmiCtx *ctx, const double *dt, const int32_t *iters, const int32_t *jiters,
                         const int32_t *flags) {
    if (!ctx) return OMI_E_ARG;
    if (!ctx->loaded) return fail(ctx, OMI_E_STATE, "no scene loaded");
    Arena &A = ctx->A;
    if (iters || flags) {
        std::vector<int> cur_it(A.W), cur_fl(A.W);
        CK(cudaMemcpy(cur_it.data(), A.w_iters, sizeof(int) * A.W, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(cur_fl.data(), A.w_flags, sizeof(int) * A.W, cudaMemcpyDeviceToHost));
        int need = 1;
        for (int w = 0; w < A.W; w++)
            need = std::max(need, passes_of(flags ? flags[w] : cur_fl[w], iters ? iters[w] : cur_it[w]));
        if (need > A.max_passes) {
            A.max_passes = need;
            const int rc0 = alloc_dynamic(ctx, A.pair_cap, A.contact_cap);
            if (rc0) return rc0;
        }
    }
    int rc = 0;
    if (dt) rc |= put(ctx, const_cast<double *>(A.w_dt), dt, A.W);
    if (iters) rc |= put(ctx, const_cast<int *>(A.w_iters), iters, A.W);
    if (jiters) rc |= put(ctx, const_cast<int *>(A.w_jiters), jiters, A.W);
    if (flags) rc |= put(ctx, const_cast<int *>(A.w_flags), flags, A.W);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_set_active(OmiCtx *ctx, const uint8_t *active) {
    if (!ctx || !active) return OMI_E_ARG;
    if (!ctx->loaded) return fail(ctx, OMI_E_STATE, "no scene loaded");
    std::memcpy(ctx->h_active.data(), active, ctx->A.W);
    CK(cudaMemcpyAsync(const_cast<uint8_t *>(ctx->A.w_active), ctx->h_active.data(), ctx->A.W,
                       cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_upload_state(OmiCtx *ctx, int32_t begin, int32_t count, const double *pos, const double *q,
                     const double *v, const double *w, const uint8_t *awake, const double *timer) {
    if (!ctx) return OMI_E_ARG;
    if (!ctx->loaded) return fail(ctx, OMI_E_STATE, "no scene loaded");
    if (begin < 0 || count < 0 || begin + count > ctx->A.NB) return fail(ctx, OMI_E_ARG, "row range");
    Arena &A = ctx->A;
    auto cp = [&](void *dst, const void *src, size_t bytes) {
        return src ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream) : cudaSuccess;
    };
    CK(cp(A.pos + (size_t)begin * 3, pos, sizeof(double) * 3 * count));
    CK(cp(A.q + (size_t)begin * 4, q, sizeof(double) * 4 * count));
    CK(cp(A.v + (size_t)begin * 3, v, sizeof(double) * 3 * count));
    CK(cp(A.w + (size_t)begin * 3, w, sizeof(double) * 3 * count));
    CK(cp(A.awake + begin, awake, count));
    CK(cp(A.timer + begin, timer, sizeof(double) * count));
    return 0;
}

int omi_download_state(OmiCtx *ctx, int32_t begin, int32_t count, double *pos, double *q, double *v,
                       double *w, uint8_t *awake, double *timer, double *amin, double *amax) {
    if (!ctx) return OMI_E_ARG;
    if (!ctx->loaded) return fail(ctx, OMI_E_STATE, "no scene loaded");
    if (begin < 0 || count < 0 || begin + count > ctx->A.NB) return fail(ctx, OMI_E_ARG, "row range");
    Arena &A = ctx->A;
    auto cp = [&](void *dst, const void *src, size_t bytes) {
        return dst ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream) : cudaSuccess;
    };
    CK(cp(pos, A.pos + (size_t)begin * 3, sizeof(double) * 3 * count));
    CK(cp(q, A.q + (size_t)begin * 4, sizeof(double) * 4 * count));
    CK(cp(v, A.v + (size_t)begin * 3, sizeof(double) * 3 * count));
    CK(cp(w, A.w + (size_t)begin * 3, sizeof(double) * 3 * count));
    CK(cp(awake, A.awake + begin, count));
    CK(cp(timer, A.timer + begin, sizeof(double) * count));
    CK(cp(amin, A.aabb_min + (size_t)begin * 3, sizeof(double) * 3 * count));
    CK(cp(amax, A.aabb_max + (size_t)begin * 3, sizeof(double) * 3 * count));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_download_joints(OmiCtx *ctx, double *la, double *lb, uint8_t *hla, uint8_t *hlb,
                        double *len, uint8_t *hlen, double *accum) {
    if (!ctx) return OMI_E_ARG;
    if (!ctx->loaded) return fail(ctx, OMI_E_STATE, "no scene loaded");
    Arena &A = ctx->A;
    const size_t J = A.NJ;
    auto cp = [&](void *dst, const void *src, size_t bytes) {
        return (dst && bytes) ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream) : cudaSuccess;
    };
    CK(cp(la, A.j_local_a, sizeof(double) * 3 * J));
    CK(cp(lb, A.j_local_b, sizeof(double) * 3 * J));
    CK(cp(hla, A.j_has_local_a, J));
    CK(cp(hlb, A.j_has_local_b, J));
    CK(cp(len, A.j_length, sizeof(double) * J));
    CK(cp(hlen, A.j_has_length, J));
    CK(cp(accum, A.j_accum, sizeof(double) * J));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_step(OmiCtx *ctx, int32_t n) {
    if (!ctx || n < 0) return OMI_E_ARG;
    return run_steps(ctx, n, true);
}

int omi_step_async(OmiCtx *ctx, int32_t n) {
    if (!ctx || n < 0) return OMI_E_ARG;
    return run_steps(ctx, n, false);
}

int omi_sync(OmiCtx *ctx) {
    if (!ctx) return OMI_E_ARG;
    int rc = read_status(ctx);
    if (rc) return rc;
    if (ctx->h_status[ST_SWEEP_TIMEOUT] || ctx->h_status[ST_BOUNDS]) return status_errors(ctx);
    if (ctx->h_status[ST_OVERFLOW])
        return fail(ctx, OMI_E_STATE, "an asynchronous step overflowed its buffers; re-run with omi_step");
    return status_errors(ctx);
}

int omi_bounds_checked(void) {
#ifdef OMI_BOUNDS_CHECK
    return 1;
#else
    return 0;
#endif
}

int omi_bounds_probe(OmiCtx *ctx, int32_t pair) {
    if (!ctx) return OMI_E_ARG;
#ifdef OMI_BOUNDS_CHECK
    if (pair < -1) return fail(ctx, OMI_E_ARG, "omi_bounds_probe: pair must be >= -1");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));     // no step of this context reads it meanwhile
    CK(cudaMemcpyToSymbol(g_bounds_probe, &pair, sizeof(int)));
    return 0;
#else
    (void)pair;
    return fail(ctx, OMI_E_UNSUPPORTED, "omi_bounds_probe: this is not the bounds-checked build");
#endif
}

int omi_set_limits(OmiCtx *ctx, int32_t spin_limit, int32_t epa_faces, int32_t stall_run) {
    if (!ctx) return OMI_E_ARG;
    if (epa_faces > EPA_F || (epa_faces > 0 && epa_faces < 4) || stall_run < -1)
        return fail(ctx, OMI_E_ARG, "limits out of range (epa_faces 4.." + std::to_string(EPA_F) + ", stall_run >= -1)");
    ctx->spin_limit = spin_limit > 0 ? spin_limit : SPIN_LIMIT_DEFAULT;
    ctx->epa_faces = epa_faces > 0 ? epa_faces : EPA_F;
    ctx->stall_run = stall_run;
    if (ctx->loaded) {
        cudaStreamSynchronize(ctx->stream);
        drop_graph(ctx);                 // the captured launches hold the arena by value
        ctx->A.spin_limit = ctx->spin_limit;
        ctx->A.epa_faces = ctx->epa_faces;
        ctx->A.stall_run = ctx->stall_run;
    }
    return 0;
}

int omi_set_tuning(OmiCtx *ctx, const OmiTuning *t) {
    if (!ctx || !t) return OMI_E_ARG;
    const bool ok = (t->sweep_warps == 4 || t->sweep_warps == 8) &&
                    (t->sweep_max_split == 1 || t->sweep_max_split == 2 || t->sweep_max_split == 4) &&
                    (t->pair_block == 128 || t->pair_block == 256 || t->pair_block == 512) &&
                    t->pair_blocks_per_sm >= 1 && t->pair_blocks_per_sm <= 32 &&
                    (t->narrow_block == 64 || t->narrow_block == 128 || t->narrow_block == 256) &&
                    (t->gjk_warps == 2 || t->gjk_warps == 4 || t->gjk_warps == 8) &&
                    t->wide_sweep_blocks >= 1 && t->wide_sweep_blocks <= 1024 &&
                    (t->wide_cluster == 0 || t->wide_cluster == 8 || t->wide_cluster == 16) &&
                    t->wide_cluster <= ctx->cluster_max &&
                    (t->sweep_claim == 8 || t->sweep_claim == 16 || t->sweep_claim == 32);
    if (!ok) return fail(ctx, OMI_E_ARG, "launch configuration out of range");
    cudaStreamSynchronize(ctx->stream);
    drop_graph(ctx);                     // re-captured with the new launches on the next step
    ctx->tune = *t;
    ctx->A.sweep_claim = t->sweep_claim;
    return 0;
}

int omi_set_wide_threshold(OmiCtx *ctx, int32_t bodies) {
    if (!ctx || bodies < 0) return OMI_E_ARG;
    ctx->wide_min_bodies = bodies;
    return 0;
}

int omi_set_cluster_budget(OmiCtx *ctx, int32_t ints) {
    if (!ctx || ints < 0) return OMI_E_ARG;
    cudaStreamSynchronize(ctx->stream);
    drop_graph(ctx);                     // the budget is a launch argument of the captured sweep
    ctx->cluster_ints = ints;
    return 0;
}

int omi_get_tuning(OmiCtx *ctx, OmiTuning *t) {
    if (!ctx || !t) return OMI_E_ARG;
    *t = ctx->tune;
    return 0;
}

int omi_validate_scene(const OmiScene *scene, char *err, int32_t err_cap) {
    SceneDerived D;
    std::string msg;
    const int rc = derive_scene(scene, D, msg);
    if (rc && err && err_cap > 0) {
        const size_t k = std::min<size_t>(msg.size(), (size_t)err_cap - 1);
        std::memcpy(err, msg.data(), k);
        err[k] = 0;
    }
    return rc;
}

// ---- stage entry points -------------------------------------------------
#define STAGE_PRELUDE                                                           \
    if (!ctx) return OMI_E_ARG;                                                 \
    if (!ctx->loaded) return fail(ctx, OMI_E_STATE, "no scene loaded");

int omi_integrate_forces(OmiCtx *ctx) {
    STAGE_PRELUDE
    k_integrate_forces<<<grid_for(ctx->A.NB, 256, SM_CAP), 256, 0, ctx->stream>>>(ctx->A, 0);
    ctx->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_refit_aabbs(OmiCtx *ctx) {
    STAGE_PRELUDE
    stage_refit(ctx, nullptr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_broadphase(OmiCtx *ctx) {
    STAGE_PRELUDE
    for (int guard = 0; guard < 16; guard++) {
        if (reset_status(ctx)) return fail(ctx, OMI_E_CUDA, "status reset");
        stage_broadphase(ctx, nullptr);
        CK(cudaGetLastError());
        int rc = read_status(ctx);
        if (rc) return rc;
        if (!ctx->h_status[ST_OVERFLOW]) return 0;
        rc = grow_for_overflow(ctx);
        if (rc) return rc;
    }
    return fail(ctx, OMI_E_STATE, "broadphase did not fit");
}

int omi_narrowphase(OmiCtx *ctx) {
    STAGE_PRELUDE
    for (int guard = 0; guard < 16; guard++) {
        if (reset_status(ctx)) return fail(ctx, OMI_E_CUDA, "status reset");
        stage_narrow(ctx, nullptr);
        stage_compact(ctx, nullptr);
        CK(cudaGetLastError());
        int rc = read_status(ctx);
        if (rc) return rc;
        if (!ctx->h_status[ST_OVERFLOW]) return 0;
        rc = grow_for_overflow(ctx);
        if (rc) return rc;
        stage_broadphase(ctx, nullptr);
    }
    return fail(ctx, OMI_E_STATE, "narrowphase did not fit");
}

int omi_solve_contacts(OmiCtx *ctx) {
    STAGE_PRELUDE
    stage_solve(ctx, nullptr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_solve_joints(OmiCtx *ctx) {
    STAGE_PRELUDE
    stage_joints(ctx, nullptr, 0);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_integrate_positions(OmiCtx *ctx) {
    STAGE_PRELUDE
    stage_finalize(ctx, FIN_POSITIONS);
    ctx->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_update_sleep(OmiCtx *ctx) {
    STAGE_PRELUDE
    stage_finalize(ctx, FIN_SLEEP);
    ctx->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

// ---- results --------------------------------------------------------------
int omi_counts(OmiCtx *ctx, int32_t *pairs, int32_t *contacts) {
    STAGE_PRELUDE
    const int W = ctx->A.W, NB = ctx->A.NB;
    std::vector<int> off(W + 1), ps(NB + 1);
    std::vector<int> hoff(ctx->A.W + 1);
    CK(cudaMemcpyAsync(hoff.data(), ctx->A.w_body_off, sizeof(int) * (W + 1), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(ps.data(), ctx->A.pair_scan, sizeof(int) * (NB + 1), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const int P = ps[NB];
    std::vector<int> cs(std::max(P, 0) + 1, 0);
    if (P >= 0 && P <= ctx->A.pair_cap)
        CK(cudaMemcpyAsync(cs.data(), ctx->A.contact_scan, sizeof(int) * (P + 1), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int w = 0; w < W; w++) {
        const int p0 = ps[hoff[w]], p1 = ps[hoff[w + 1]];
        if (pairs) pairs[w] = p1 - p0;
        if (contacts) contacts[w] = cs[p1] - cs[p0];
    }
    return 0;
}

static int world_ranges(OmiCtx *ctx, int w, int &p0, int &p1, int &c0, int &c1) {
    int bo[2];
    CK(cudaMemcpyAsync(bo, ctx->A.w_body_off + w, sizeof(int) * 2, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpyAsync(&p0, ctx->A.pair_scan + bo[0], sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&p1, ctx->A.pair_scan + bo[1], sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpyAsync(&c0, ctx->A.contact_scan + p0, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&c1, ctx->A.contact_scan + p1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_get_pairs(OmiCtx *ctx, int32_t w, int32_t *out, int32_t cap) {
    int rc = check_world(ctx, w);
    if (rc) return rc;
    int p0, p1, c0, c1;
    rc = world_ranges(ctx, w, p0, p1, c0, c1);
    if (rc) return rc;
    const int n = p1 - p0;
    if (n > cap) return fail(ctx, OMI_E_ARG, "pair buffer too small");
    std::vector<int> a(n), b(n);
    if (n) {
        CK(cudaMemcpyAsync(a.data(), ctx->A.pair_a + p0, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(b.data(), ctx->A.pair_b + p0, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    for (int i = 0; i < n; i++) { out[2 * i] = a[i]; out[2 * i + 1] = b[i]; }
    return n;
}

int omi_get_contacts(OmiCtx *ctx, int32_t w, int32_t *a, int32_t *b, double *pt, double *nrm,
                     double *depth, double *imp, int32_t cap) {
    int rc = check_world(ctx, w);
    if (rc) return rc;
    int p0, p1, c0, c1;
    rc = world_ranges(ctx, w, p0, p1, c0, c1);
    if (rc) return rc;
    const int n = c1 - c0;
    if (n > cap) return fail(ctx, OMI_E_ARG, "contact buffer too small");
    Arena &A = ctx->A;
    auto cp = [&](void *dst, const void *src, size_t bytes) {
        return (dst && bytes) ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream) : cudaSuccess;
    };
    CK(cp(a, A.c_a + c0, sizeof(int) * n));
    CK(cp(b, A.c_b + c0, sizeof(int) * n));
    CK(cp(pt, A.c_pt + (size_t)c0 * 3, sizeof(double) * 3 * n));
    CK(cp(nrm, A.c_n + (size_t)c0 * 3, sizeof(double) * 3 * n));
    CK(cp(depth, A.c_depth + c0, sizeof(double) * n));
    CK(cp(imp, A.c_imp + (size_t)c0 * 3, sizeof(double) * 3 * n));
    int flags = 0;
    CK(cudaMemcpyAsync(&flags, A.w_flags + w, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // the reference writes the solved impulses back to its contacts only with
    // warm start on (solver.py:271-278); otherwise they stay zero
    if (imp && !(flags & OMI_WF_WARM)) std::fill(imp, imp + (size_t)3 * n, 0.0);
    return n;
}

int omi_get_trigger_overlaps(OmiCtx *ctx, int32_t w, int32_t *trg, int32_t *other, int32_t cap) {
    int rc = check_world(ctx, w);
    if (rc) return rc;
    if (cap < 0 || (cap > 0 && (!trg || !other))) return fail(ctx, OMI_E_ARG, "null output or negative cap");
    if (!ctx->has_triggers) return 0;
    CK(cudaStreamSynchronize(ctx->stream));
    int n = 0;
    CK(cudaMemcpy(&n, ctx->A.trig_n, sizeof(int), cudaMemcpyDeviceToHost));
    n = std::min(n, ctx->A.pair_cap);
    std::vector<int> out((size_t)n * 3);
    if (n) CK(cudaMemcpy(out.data(), ctx->A.trig_out, sizeof(int) * 3 * n, cudaMemcpyDeviceToHost));
    const int b0 = ctx->h_body_off[w], b1 = b0 + ctx->h_body_n[w];
    std::vector<std::pair<int, int>> hits;
    for (int k = 0; k < n; k++) {
        const int t = out[k * 3], o = out[k * 3 + 1];
        if (out[k * 3 + 2] == 1 && t >= b0 && t < b1) hits.emplace_back(t - b0, o - b0);
    }
    std::sort(hits.begin(), hits.end());
    const int m = (int)hits.size();
    for (int k = 0; k < std::min(m, (int)cap); k++) { trg[k] = hits[k].first; other[k] = hits[k].second; }
    return m;
}

int omi_world_levels(OmiCtx *ctx, int32_t *levels) {
    STAGE_PRELUDE
    if (!levels) return fail(ctx, OMI_E_ARG, "null output");
    CK(cudaMemcpyAsync(levels, ctx->A.w_levels, sizeof(int) * ctx->A.W, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_get_islands(OmiCtx *ctx, int32_t w, int32_t *labels) {
    int rc = check_world(ctx, w);
    if (rc) return rc;
    int bo[2];
    CK(cudaMemcpyAsync(bo, ctx->A.w_body_off + w, sizeof(int) * 2, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpyAsync(labels, ctx->A.b_island + bo[0], sizeof(int) * (bo[1] - bo[0]), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_get_cache(OmiCtx *ctx, int32_t w, int32_t *a, int32_t *b, double *pt, double *imp,
                  int32_t cap) {
    int rc = check_world(ctx, w);
    if (rc) return rc;
    Arena &A = ctx->A;
    int cur = 0, off = 0, n = 0;
    CK(cudaMemcpyAsync(&cur, A.parity, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpyAsync(&off, A.w_cache_off[cur] + w, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&n, A.w_cache_n[cur] + w, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (n > cap) return fail(ctx, OMI_E_ARG, "cache buffer too small");
    auto cp = [&](void *dst, const void *src, size_t bytes) {
        return (dst && bytes) ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream) : cudaSuccess;
    };
    CK(cp(a, A.cache_a[cur] + off, sizeof(int) * n));
    CK(cp(b, A.cache_b[cur] + off, sizeof(int) * n));
    CK(cp(pt, A.cache_pt[cur] + (size_t)off * 3, sizeof(double) * 3 * n));
    CK(cp(imp, A.cache_imp[cur] + (size_t)off * 3, sizeof(double) * 3 * n));
    CK(cudaStreamSynchronize(ctx->stream));
    return n;
}

int omi_set_cache(OmiCtx *ctx, int32_t w, int32_t n, const int32_t *a, const int32_t *b,
                  const double *pt, const double *imp) {
    int rc = check_world(ctx, w);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!a || !b || !pt || !imp))) return fail(ctx, OMI_E_ARG, "cache arrays");
    Arena &A = ctx->A;
    const int W = A.W;
    for (int i = 0; i < n; i++)
        if (a[i] < 0 || a[i] >= A.NB || b[i] < 0 || b[i] >= A.NB) return fail(ctx, OMI_E_ARG, "cache body index");
    CK(cudaStreamSynchronize(ctx->stream));
    int cur = 0;
    CK(cudaMemcpy(&cur, A.parity, sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> off(W), cnt(W);
    CK(cudaMemcpy(off.data(), A.w_cache_off[cur], sizeof(int) * W, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cnt.data(), A.w_cache_n[cur], sizeof(int) * W, cudaMemcpyDeviceToHost));
    // gather every world's entries, replace world w's, lay them out again
    std::vector<int> ha, hb;
    std::vector<double> hp, hi;
    std::vector<int> noff(W), ncnt(W);
    for (int v = 0; v < W; v++) {
        noff[v] = (int)ha.size();
        if (v == w) {
            ha.insert(ha.end(), a, a + n); hb.insert(hb.end(), b, b + n);
            hp.insert(hp.end(), pt, pt + 3 * n); hi.insert(hi.end(), imp, imp + 3 * n);
            ncnt[v] = n;
            continue;
        }
        const int m = cnt[v], o = off[v];
        const size_t base = ha.size();
        ha.resize(base + m); hb.resize(base + m); hp.resize((base + m) * 3); hi.resize((base + m) * 3);
        if (m) {
            CK(cudaMemcpy(&ha[base], A.cache_a[cur] + o, sizeof(int) * m, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(&hb[base], A.cache_b[cur] + o, sizeof(int) * m, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(&hp[base * 3], A.cache_pt[cur] + (size_t)o * 3, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(&hi[base * 3], A.cache_imp[cur] + (size_t)o * 3, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost));
        }
        ncnt[v] = m;
    }
    const int total = (int)ha.size();
    if (total > ctx->cache_cap) {
        const int want = total;
        rc = alloc_dynamic(ctx, std::max(ctx->A.pair_cap, want), std::max(ctx->A.contact_cap, want));
        if (rc) return rc;
    }
    if (total) {
        CK(cudaMemcpy(A.cache_a[cur], ha.data(), sizeof(int) * total, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(A.cache_b[cur], hb.data(), sizeof(int) * total, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(A.cache_pt[cur], hp.data(), sizeof(double) * 3 * total, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(A.cache_imp[cur], hi.data(), sizeof(double) * 3 * total, cudaMemcpyHostToDevice));
    }
    CK(cudaMemcpy(A.w_cache_off[cur], noff.data(), sizeof(int) * W, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(A.w_cache_n[cur], ncnt.data(), sizeof(int) * W, cudaMemcpyHostToDevice));
    CK(cudaMemset(A.hkey[cur], 0xff, sizeof(unsigned long long) * ((size_t)A.hash_mask + 1)));
    CK(cudaMemset(A.hused_n + cur, 0, sizeof(int)));
    k_hash_rebuild<<<std::min(W, 65535), 128, 0, ctx->stream>>>(A, cur);
    ctx->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int omi_profile_step(OmiCtx *ctx, float *ms, int32_t n, int32_t *n_out) {
    STAGE_PRELUDE
    Prof pf;
    pf.on = true;
    for (int i = 0; i <= KN_COUNT; i++) CK(cudaEventCreate(&pf.ev[i]));
    for (int guard = 0; guard < 16; guard++) {
        if (reset_status(ctx)) return fail(ctx, OMI_E_CUDA, "status reset");
        enqueue_step(ctx, &pf);
        CK(cudaGetLastError());
        int rc = read_status(ctx);
        if (rc) return rc;
        if (ctx->h_status[ST_STEPS_DONE] == 1) break;
        rc = grow_for_overflow(ctx);
        if (rc) return rc;
    }
    ctx->prof_ms.assign(KN_COUNT, 0.0f);
    for (int k = 0; k < KN_COUNT; k++) {
        float t = 0.0f;
        cudaEventElapsedTime(&t, pf.ev[k], pf.ev[k + 1]);
        ctx->prof_ms[k] = t;
    }
    for (int i = 0; i <= KN_COUNT; i++) cudaEventDestroy(pf.ev[i]);
    const int m = std::min<int>(n, KN_COUNT);
    for (int k = 0; k < m; k++) ms[k] = ctx->prof_ms[k];
    if (n_out) *n_out = KN_COUNT;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Capsule against triangles (omi_capsule_triangles*)
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t CT_CHUNK = int64_t(1) << 21;   // triangles per pipelined chunk (~270 MB a buffer set)

int capsule_grid(OmiCtx *ctx, int64_t n) {
    if (!ctx->cap_blocks) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_capsule_triangles, CT_THREADS, 0) != cudaSuccess ||
            b < 1)
            b = 1;
        ctx->cap_blocks = b;
    }
    const int64_t tiles = (n + CT_THREADS - 1) / CT_THREADS;
    return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)ctx->sm_count * ctx->cap_blocks));
}

int capsule_check(OmiCtx *ctx, int32_t q, int64_t n, const void *caps, const void *tri_off, const void *verts,
                  const void *hit, const void *points, const void *normals, const void *depths) {
    if (!ctx) return OMI_E_ARG;
    if (n < 0) return fail(ctx, OMI_E_ARG, "negative triangle count");
    if (n > 0 && q < 1) return fail(ctx, OMI_E_ARG, "triangles without a capsule");
    if (q < 0) return fail(ctx, OMI_E_ARG, "negative capsule count");
    if (n > 0 && (!caps || !tri_off || !verts || !hit || !points || !normals || !depths))
        return fail(ctx, OMI_E_ARG, "null buffer");
    return 0;
}

// buffers for q capsules and chunks of `chunk` triangles (regrown, never shrunk)
int capsule_buffers(OmiCtx *ctx, int32_t q, int64_t chunk) {
    if (!ctx->cap_s[0]) {
        for (int k = 0; k < 2; k++) CK(cudaStreamCreateWithFlags(&ctx->cap_s[k], cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->cap_ev, cudaEventDisableTiming));
    }
    if (q <= ctx->cap_q && chunk <= ctx->cap_chunk) return 0;
    for (int k = 0; k < 2; k++) CK(cudaStreamSynchronize(ctx->cap_s[k]));
    CK(cudaStreamSynchronize(ctx->stream));
    free_pool(ctx, ctx->capbufs);
    ctx->cap_q = std::max(q, ctx->cap_q);
    ctx->cap_chunk = std::max(chunk, ctx->cap_chunk);
    int rc = alloc(ctx, ctx->capbufs, ctx->cap_caps, (size_t)ctx->cap_q * CT_CAP_DOUBLES);
    rc = rc ? rc : alloc(ctx, ctx->capbufs, ctx->cap_off, (size_t)ctx->cap_q + 1);
    for (int k = 0; k < 2 && !rc; k++) {
        const size_t m = (size_t)ctx->cap_chunk;
        rc = alloc(ctx, ctx->capbufs, ctx->cap_v[k], m * 9);
        rc = rc ? rc : alloc(ctx, ctx->capbufs, ctx->cap_h[k], m);
        rc = rc ? rc : alloc(ctx, ctx->capbufs, ctx->cap_p[k], m * 3);
        rc = rc ? rc : alloc(ctx, ctx->capbufs, ctx->cap_n[k], m * 3);
        rc = rc ? rc : alloc(ctx, ctx->capbufs, ctx->cap_d[k], m);
    }
    if (rc) { free_pool(ctx, ctx->capbufs); ctx->cap_q = 0; ctx->cap_chunk = 0; }
    return rc;
}

int capsule_pipeline(OmiCtx *ctx, int32_t q, const double *caps, const int64_t *tri_off, const double *verts,
                     int64_t n, uint8_t *hit, double *points, double *normals, double *depths) {
    int rc = capsule_check(ctx, q, n, caps, tri_off, verts, hit, points, normals, depths);
    if (rc || n == 0) return rc;
    if (tri_off[0] != 0 || tri_off[q] != n) return fail(ctx, OMI_E_ARG, "tri_off must run from 0 to n");
    for (int c = 0; c < q; c++)
        if (tri_off[c + 1] < tri_off[c]) return fail(ctx, OMI_E_ARG, "tri_off must be non-decreasing");
    const int64_t chunk = std::min<int64_t>(CT_CHUNK, (n + CT_THREADS - 1) / CT_THREADS * CT_THREADS);
    rc = capsule_buffers(ctx, q, chunk);
    if (rc) return rc;
    cudaStream_t s0 = ctx->cap_s[0], s1 = ctx->cap_s[1];
    // after the caller's earlier work on the context stream
    CK(cudaEventRecord(ctx->cap_ev, ctx->stream));
    CK(cudaStreamWaitEvent(s0, ctx->cap_ev, 0));
    CK(cudaMemcpyAsync(ctx->cap_caps, caps, sizeof(double) * CT_CAP_DOUBLES * q, cudaMemcpyHostToDevice, s0));
    CK(cudaMemcpyAsync(ctx->cap_off, tri_off, sizeof(int64_t) * (q + 1), cudaMemcpyHostToDevice, s0));
    CK(cudaEventRecord(ctx->cap_ev, s0));
    CK(cudaStreamWaitEvent(s1, ctx->cap_ev, 0));
    int k = 0;
    for (int64_t t0 = 0; t0 < n; t0 += ctx->cap_chunk, k ^= 1) {
        const int64_t m = std::min<int64_t>(ctx->cap_chunk, n - t0);
        cudaStream_t s = ctx->cap_s[k];
        CK(cudaMemcpyAsync(ctx->cap_v[k], verts + t0 * 9, sizeof(double) * 9 * m, cudaMemcpyHostToDevice, s));
        k_capsule_triangles<<<capsule_grid(ctx, m), CT_THREADS, 0, s>>>(
            ctx->cap_caps, ctx->cap_off, q, ctx->cap_v[k], t0, m, ctx->cap_h[k], ctx->cap_p[k], ctx->cap_n[k],
            ctx->cap_d[k]);
        CK(cudaGetLastError());
        ctx->launches++;
        CK(cudaMemcpyAsync(hit + t0, ctx->cap_h[k], m, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(points + t0 * 3, ctx->cap_p[k], sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(normals + t0 * 3, ctx->cap_n[k], sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(depths + t0, ctx->cap_d[k], sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s0));
    CK(cudaStreamSynchronize(s1));
    return 0;
}

}  // namespace

extern "C" {

int omi_capsule_triangles(OmiCtx *ctx, const double *p0, const double *p1, double radius, const double *verts,
                          int64_t n, uint8_t *hit, double *points, double *normals, double *depths) {
    if (!ctx) return OMI_E_ARG;
    if (!p0 || !p1) return fail(ctx, OMI_E_ARG, "null capsule end");
    const double cap[CT_CAP_DOUBLES] = {p0[0], p0[1], p0[2], p1[0], p1[1], p1[2], radius};
    const int64_t off[2] = {0, n};
    return capsule_pipeline(ctx, 1, cap, off, verts, n, hit, points, normals, depths);
}

int omi_capsule_triangles_batch(OmiCtx *ctx, int32_t q, const double *caps, const int64_t *tri_off,
                                const double *verts, int64_t n, uint8_t *hit, double *points, double *normals,
                                double *depths) {
    if (ctx && q >= 0 && !tri_off) return fail(ctx, OMI_E_ARG, "null tri_off");
    return capsule_pipeline(ctx, q, caps, tri_off, verts, n, hit, points, normals, depths);
}

int omi_capsule_triangles_device(OmiCtx *ctx, int32_t q, const double *caps, const int64_t *tri_off,
                                 const double *verts, int64_t n, uint8_t *hit, double *points, double *normals,
                                 double *depths) {
    int rc = capsule_check(ctx, q, n, caps, tri_off, verts, hit, points, normals, depths);
    if (rc || n == 0) return rc;
    k_capsule_triangles<<<capsule_grid(ctx, n), CT_THREADS, 0, ctx->stream>>>(caps, tri_off, q, verts, 0, n, hit,
                                                                              points, normals, depths);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free sweep-and-prune (omi_sweep_pairs_noalloc)
//
// For callers that cannot allocate device memory. Its scratch is this fixed
// file-scope device array; in host code `g_noalloc_scratch` is only a host-side
// stand-in for the symbol, so its device address is looked up with
// cudaGetSymbolAddress (once per device) and that address is what the kernels
// receive. Reuses the arena's sort, window-count and scan kernels through an
// Arena whose pointers all lie in the array or in the caller's buffers.
// ---------------------------------------------------------------------------
namespace {

constexpr int NA_MAX = OMI_NOALLOC_MAX_BODIES;
constexpr size_t NA_TILES = NA_MAX / SCAN_TILE + 2;
// layout (bytes), each block 256-aligned
constexpr size_t na_align(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t NA_OFF_SORTK0 = 0;
constexpr size_t NA_OFF_SORTK1 = NA_OFF_SORTK0 + na_align(sizeof(double) * NA_MAX);
constexpr size_t NA_OFF_SORTV0 = NA_OFF_SORTK1 + na_align(sizeof(double) * NA_MAX);
constexpr size_t NA_OFF_SORTV1 = NA_OFF_SORTV0 + na_align(sizeof(int) * NA_MAX);
constexpr size_t NA_OFF_ORDER = NA_OFF_SORTV1 + na_align(sizeof(int) * NA_MAX);
constexpr size_t NA_OFF_SORTX = NA_OFF_ORDER + na_align(sizeof(int) * NA_MAX);
constexpr size_t NA_OFF_CNT = NA_OFF_SORTX + na_align(sizeof(double) * NA_MAX);
constexpr size_t NA_OFF_SCAN = NA_OFF_CNT + na_align(sizeof(int) * NA_MAX);
constexpr size_t NA_OFF_ZERO = NA_OFF_SCAN + na_align(sizeof(int) * (NA_MAX + 1));   // body_world / filter rows
constexpr size_t NA_OFF_TILES = NA_OFF_ZERO + na_align(sizeof(int) * NA_MAX);
constexpr size_t NA_OFF_WORLD = NA_OFF_TILES + na_align(sizeof(int) * (NA_TILES + 1));
// world tables: body_off[2], body_n[1], flags[1], filter_off[1], filter_rows[1], active byte, filter byte
constexpr size_t NA_BYTES = NA_OFF_WORLD + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// Per-device address of the array, looked up on the first call on that
// device. Host threads calling at once are serialised by the mutex during
// that set-up only; afterwards the ready flag (acquire) guards the address.
// cudaDeviceReset on a device ends the context the address belongs to: call
// omi_sweep_pairs_noalloc on that device only in the context it was set up in.
struct NaDevice {
    std::atomic<bool> ready{false};
    unsigned char *base = nullptr;
};
NaDevice g_na_dev[64];
std::mutex g_na_setup;

void na_err(char *err, int cap, const std::string &msg) {
    if (err && cap > 0) {
        std::snprintf(err, (size_t)cap, "%s", msg.c_str());
    }
}

// world table and zeroed per-row arrays for a one-world arena of n rows
__global__ void k_noalloc_init(unsigned char *base, int n, int filter_rows, int own_filter) {
    int *world = reinterpret_cast<int *>(base + NA_OFF_WORLD);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        world[0] = 0;                 // body_off[0]
        world[1] = n;                 // body_off[1]
        world[2] = n;                 // body_n
        world[3] = WF_COLLISION;      // flags
        world[4] = 0;                 // filter_off
        world[5] = filter_rows;       // filter_rows
        base[NA_OFF_WORLD + 24] = 1;  // active
        base[NA_OFF_WORLD + 25] = 1;  // default filter matrix: everything collides
    }
    int *zero = reinterpret_cast<int *>(base + NA_OFF_ZERO);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) zero[i] = 0;
    (void)own_filter;
}

// write pairs in the reference's order into the caller's interleaved buffer
__global__ void k_noalloc_emit(Arena A, int *pairs, int cap, int *n_pairs) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_pairs = A.pair_scan[A.NB];
    for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.NB; e += nwarps) {
        const int a = A.order[e];
        const int endk = window_end(A, 0, A.NB, A.aabb_max[a * 3]);
        int out = A.pair_scan[e];
        for (int base = e + 1; base < endk; base += 32) {
            const int kj = base + lane;
            int b = -1;
            bool keep = false;
            if (kj < endk) { b = A.order[kj]; keep = pair_keep(A, 0, a, b); }
            const unsigned m = __ballot_sync(FULL, keep);
            if (keep) {
                const int slot = out + __popc(m & ((1u << lane) - 1u));
                if (slot < cap) {
                    pairs[2 * slot] = a < b ? a : b;
                    pairs[2 * slot + 1] = a < b ? b : a;
                }
            }
            out += __popc(m);
        }
    }
}

}  // namespace

extern "C" int omi_sweep_pairs_noalloc(const double *aabb_min, const double *aabb_max,
                                       const int32_t *motion_type, const int32_t *filter_row,
                                       const uint8_t *filter_matrix, int32_t filter_rows,
                                       int32_t n, int32_t *pairs, int32_t pair_cap,
                                       int32_t *n_pairs, void *stream_v, char *err,
                                       int32_t err_cap) {
    if (n < 0 || n > NA_MAX) {
        na_err(err, err_cap, "omi_sweep_pairs_noalloc: " + std::to_string(n) +
                                 " bodies exceeds the fixed scratch limit of " +
                                 std::to_string(NA_MAX) + " (OMI_NOALLOC_MAX_BODIES)");
        return OMI_E_ARG;
    }
    if (!aabb_min || !aabb_max || !motion_type || !n_pairs || pair_cap < 0 || (pair_cap > 0 && !pairs)) {
        na_err(err, err_cap, "omi_sweep_pairs_noalloc: null buffer or negative pair_cap");
        return OMI_E_ARG;
    }
    if ((filter_row == nullptr) != (filter_matrix == nullptr) || (filter_row && filter_rows < 1)) {
        na_err(err, err_cap, "omi_sweep_pairs_noalloc: filter_row and filter_matrix go together");
        return OMI_E_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        na_err(err, err_cap, std::string("omi_sweep_pairs_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return OMI_E_CUDA;
    }
    NaDevice &nd = g_na_dev[dev];
    if (!nd.ready.load(std::memory_order_acquire)) {   // set-up, once per device, with that device current
        std::lock_guard<std::mutex> lock(g_na_setup);
        if (!nd.ready.load(std::memory_order_relaxed)) {
            void *addr = nullptr;
            e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess || !addr) {
                na_err(err, err_cap, std::string("omi_sweep_pairs_noalloc: cudaGetSymbolAddress: ") +
                                         cudaGetErrorString(e));
                return OMI_E_CUDA;
            }
            e = cudaFuncSetAttribute(k_sort<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * 24);
            if (e != cudaSuccess) {
                na_err(err, err_cap, std::string("omi_sweep_pairs_noalloc: cudaFuncSetAttribute: ") +
                                         cudaGetErrorString(e));
                return OMI_E_CUDA;
            }
            nd.base = static_cast<unsigned char *>(addr);
            nd.ready.store(true, std::memory_order_release);
        }
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream_v);
    unsigned char *base = nd.base;
    int *world = reinterpret_cast<int *>(base + NA_OFF_WORLD);
    Arena A{};
    A.W = 1;
    A.NB = n;
    A.pair_cap = pair_cap;
    A.w_body_off = world;
    A.w_body_n = world + 2;
    A.w_flags = world + 3;
    A.w_filter_off = world + 4;
    A.w_filter_rows = world + 5;
    A.w_active = base + NA_OFF_WORLD + 24;
    A.body_world = reinterpret_cast<int *>(base + NA_OFF_ZERO);
    A.aabb_min = const_cast<double *>(aabb_min);
    A.aabb_max = const_cast<double *>(aabb_max);
    A.mtype = motion_type;
    A.filter_row = filter_row ? filter_row : reinterpret_cast<int *>(base + NA_OFF_ZERO);
    A.filter_matrix = filter_matrix ? filter_matrix : base + NA_OFF_WORLD + 25;
    A.sort_k[0] = reinterpret_cast<double *>(base + NA_OFF_SORTK0);
    A.sort_k[1] = reinterpret_cast<double *>(base + NA_OFF_SORTK1);
    A.sort_v[0] = reinterpret_cast<int *>(base + NA_OFF_SORTV0);
    A.sort_v[1] = reinterpret_cast<int *>(base + NA_OFF_SORTV1);
    A.order = reinterpret_cast<int *>(base + NA_OFF_ORDER);
    A.sorted_x = reinterpret_cast<double *>(base + NA_OFF_SORTX);
    A.pair_cnt = reinterpret_cast<int *>(base + NA_OFF_CNT);
    A.pair_scan = reinterpret_cast<int *>(base + NA_OFF_SCAN);
    int *tiles = reinterpret_cast<int *>(base + NA_OFF_TILES);
    const int rows = filter_row ? filter_rows : 1;
    k_noalloc_init<<<grid_for(std::max(n, 1), 256, 64), 256, 0, st>>>(base, n, rows, filter_row != nullptr);
    const int sort_cap = std::min(std::max(n, 1), 8192);
    k_sort<false><<<1, n > 2048 ? 1024 : 256, (size_t)sort_cap * 24, st>>>(A, sort_cap);
    k_pair_count_boxes<<<grid_for(std::max(n, 1) * 32, 256, 148 * 16), 256, 0, st>>>(A);
    const int ntiles = std::max(1, (n + SCAN_TILE - 1) / SCAN_TILE);
    k_scan_tiles<<<ntiles, 1024, 0, st>>>(A.pair_cnt, A.pair_scan, n, nullptr, nullptr, 0, 0, tiles);
    k_scan_top<<<1, 1024, 0, st>>>(tiles, ntiles, nullptr, 0, 0);
    k_scan_add<<<ntiles, 1024, 0, st>>>(A.pair_scan, n, nullptr, tiles, ntiles, nullptr, 0, 0);
    k_noalloc_emit<<<grid_for(std::max(n, 1) * 32, 256, 148 * 16), 256, 0, st>>>(A, pairs, pair_cap, n_pairs);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        na_err(err, err_cap, std::string("omi_sweep_pairs_noalloc: launch: ") + cudaGetErrorString(e));
        return OMI_E_CUDA;
    }
    return 0;
}
