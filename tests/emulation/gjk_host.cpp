// The device GJK/EPA (omi_physics_b200/csrc/gjk.cuh) compiled for the host
// with one lane per warp, so the CPU test suite can compare it with the
// oracle's restatement (or_collide_convex) pair by pair. Test infrastructure:
// the CUDA builtins the header uses are stood in for by their one-lane
// meaning (a shuffle returns the lane's own value).
#include <cmath>
#include <cstdint>
#define __device__
#define __forceinline__ inline
struct TI { unsigned x = 0; };
static TI threadIdx;
static inline double __shfl_xor_sync(unsigned, double x, int) { return x; }
static inline int __shfl_sync(unsigned, int x, int) { return x; }
static inline void __syncwarp() {}
#define OMI_HOST_EMULATION
#include "../../omi_physics_b200/csrc/gjk.cuh"
using namespace omi;
static EpaWork W;
extern "C" int emu_collide(int ka, const double *ca, const double *qa, const double *sa, double ra, const double *pa, int ma,
                           int kb, const double *cb, const double *qb, const double *sb, double rb, const double *pb, int mb,
                           double *nrm, double *pt, double *dep) {
    Proxy P[2];
    const int ks[2] = {ka, kb}; const double *cs[2] = {ca, cb}, *qs[2] = {qa, qb}, *ss[2] = {sa, sb}, *ps[2] = {pa, pb};
    const double rs[2] = {ra, rb}; const int ms[2] = {ma, mb};
    for (int e = 0; e < 2; e++) {
        Proxy &p = P[e];
        p.kind = ks[e];
        quat_to_matrix(qs[e], p.R);
        for (int c = 0; c < 3; c++) { p.c[c] = cs[e][c]; p.h[c] = 0.5 * ss[e][c]; }
        p.r = rs[e]; p.local = ps[e]; p.m = ms[e];
        if (p.kind == 4) capsule_ends(p.c, p.R, 0.5 * ss[e][1], p.e0, p.e1);
    }
    *dep = 0.0;
    return collide_convex(P[0], P[1], W, nrm, pt, dep);
}
