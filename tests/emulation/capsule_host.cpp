// The device capsule-against-triangle arithmetic (omi_physics_b200/csrc/
// capsule.cuh) compiled for the host, so the CPU test suite can compare it
// with the oracle's restatement (or_capsule_triangles) triangle by triangle.
// Test infrastructure only.
#include <cmath>
#include <cstdint>
#define __device__
#define __forceinline__ inline
#define OMI_HOST_EMULATION
#include "../../omi_physics_b200/csrc/capsule.cuh"
using namespace omi;

extern "C" void emu_capsule_triangles(const double *c0, const double *c1, double radius, const double *verts,
                                      int64_t n, uint8_t *hit, double *points, double *normals, double *depths) {
    double centre[3];
    for (int k = 0; k < 3; k++) centre[k] = (c0[k] + c1[k]) * 0.5;
    for (int64_t i = 0; i < n; i++) {
        const double *v = verts + i * 9;
        double pt[3], nr[3], dep;
        const int h = capsule_triangle(c0, c1, centre, radius, v, v + 3, v + 6, pt, nr, &dep);
        hit[i] = (uint8_t)h;
        if (h) {
            for (int k = 0; k < 3; k++) { points[i * 3 + k] = pt[k]; normals[i * 3 + k] = nr[k]; }
            depths[i] = dep;
        }
    }
}
