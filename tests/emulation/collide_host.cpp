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

extern "C" int emu_sphere_sphere(const double *ca, double ra, const double *cb, double rb, double *normal,
                                 double *pts, double *deps) {
    return sphere_sphere(ca, ra, cb, rb, normal, pts, deps);
}

extern "C" int emu_sphere_box(const double *cs, double rs, const double *cb, const double *Rb, const double *hb,
                              double *normal, double *pts, double *deps) {
    return sphere_box(cs, rs, cb, Rb, hb, normal, pts, deps);
}

extern "C" void emu_quat_to_matrix(const double *q, double *R) { quat_to_matrix(q, R); }
