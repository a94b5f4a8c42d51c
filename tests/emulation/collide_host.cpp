// The device narrowphase primitives (omi_physics_b200/csrc/geometry.cuh:
// box-box SAT + face clipping + reduction, sphere-sphere, sphere-box, and the
// quaternion-to-matrix conversion the step runs on every body) compiled for
// the host, so the CPU test suite can compare them with the oracle's
// restatements pair by pair. Test infrastructure only.
#include <cmath>
#include <cstdint>
#define __device__
#define __forceinline__ inline
#define OMI_HOST_EMULATION
#include "../../omi_physics_b200/csrc/geometry.cuh"
using namespace omi;

extern "C" int emu_box_box(const double *ca, const double *Ra, const double *ha, const double *cb,
                           const double *Rb, const double *hb, double *normal, double *pts, double *deps) {
    return box_box(ca, Ra, ha, cb, Rb, hb, normal, pts, deps);
}

// the step's form of the same test: k_narrow runs the six face axes and
// leaves its best axis in the pair's slot; k_edge_clip reads it back, runs
// the nine edge axes and clips the touching pairs
extern "C" int emu_box_box_split(const double *ca, const double *Ra, const double *ha, const double *cb,
                                 const double *Rb, const double *hb, double *normal, double *pts, double *deps) {
    SatBest best;
    sat_begin(best);
    if (!sat_axes(0, 6, ca, Ra, ha, cb, Rb, hb, best)) return 0;
    double slot[4] = {best.x, best.y, best.z, best.depth};
    SatBest resumed;
    resumed.x = slot[0]; resumed.y = slot[1]; resumed.z = slot[2]; resumed.depth = slot[3];
    if (!sat_axes(6, 15, ca, Ra, ha, cb, Rb, hb, resumed)) return 0;
    normal[0] = resumed.x; normal[1] = resumed.y; normal[2] = resumed.z;
    return clip_faces(ca, Ra, ha, cb, Rb, hb, normal, resumed.depth, pts, deps);
}

extern "C" int emu_sphere_sphere(const double *ca, double ra, const double *cb, double rb, double *normal,
                                 double *pts, double *deps) {
    return sphere_sphere(ca, ra, cb, rb, normal, pts, deps);
}

extern "C" int emu_sphere_box(const double *cs, double rs, const double *cb, const double *Rb, const double *hb,
                              double *normal, double *pts, double *deps) {
    return sphere_box(cs, rs, cb, Rb, hb, normal, pts, deps);
}

extern "C" void emu_quat_to_matrix(const double *q, double *R) { quat_to_matrix(q, R); }
