// angle_metrics.cuh -- the reference's angle criteria (QualityCriterium::MIN_ANGLE / MAX_ANGLE)
// for triangles in the plane, triangles on a surface and tetrahedra, as device functions.
//
//   minAngleMetricTri2D / maxAngleMetricTri2D   dmo/DMOQualityTri.h:10-29, 124-144
//   minAngleMetricTri(p, n) / maxAngleMetricTri  dmo/DMOQualityTri.h:50-71, 166-189
//   minAngleMetricTet / maxAngleMetricTet        dmo/DMOQualityTet.h:10-37, 62-91
//   calcAngle                                    dmo/DMOQualityUtil.h:30-50
// min angle: q = 3 min_angle / pi (1 for the equilateral triangle; for a tet the smallest
// dihedral angle, 3 acos(1/3) / pi = 1.175 for the regular tet); max angle: q = 1 - max / pi.
// A flipped element returns its signed area / volume, like the reference. The division by pi
// is done in double as the reference's `/ M_PI` does. Angles come from acosf (CUDA's); since
// acos decreases, the minimum (maximum) of the angles is taken as acosf of the largest
// (smallest) cosine: one acosf per element instead of three or six.
#pragma once
#include <cfloat>

namespace vsdmo {

constexpr double ANG_PI = 3.14159265358979323846;

// cosine of the angle between u and v: dot / sqrt(|u|^2 |v|^2) (calcAngle before its acos)
__host__ __device__ __forceinline__ float ang_cos2(float ux, float uy, float vx, float vy) {
    const float d = ux * vx + uy * vy;
    return d / sqrtf((ux * ux + uy * uy) * (vx * vx + vy * vy));
}
__host__ __device__ __forceinline__ float ang_cos3(const float* u, const float* v) {
    const float d = (u[0] * v[0] + u[1] * v[1]) + u[2] * v[2];
    return d / sqrtf(((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]) * ((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]));
}

template <bool MAXA>
__device__ __forceinline__ float angle_q(float cmax, float cmin) {
    if (MAXA) return 1.f - (float)((double)acosf(cmin) / ANG_PI);
    return (float)((double)(3.f * acosf(cmax)) / ANG_PI);
}

// triangle (a, b, c) in the plane
template <bool MAXA>
__device__ __forceinline__ float tri2d_angle(float ax, float ay, float bx, float by, float cx, float cy) {
    const float e0x = bx - ax, e0y = by - ay, e1x = cx - bx, e1y = cy - by;
    const float area = e0x * e1y - e0y * e1x;
    if (area < 0.f) return area;
    // angles at b (a-b, c-b), at c (b-c, a-c), at a (c-a, b-a)
    const float c1 = ang_cos2(ax - bx, ay - by, cx - bx, cy - by);
    const float c2 = ang_cos2(bx - cx, by - cy, ax - cx, ay - cy);
    const float c3 = ang_cos2(cx - ax, cy - ay, bx - ax, by - ay);
    return angle_q<MAXA>(fmaxf(fmaxf(c1, c2), c3), fminf(fminf(c1, c2), c3));
}

// triangle (p0, p1, p2) in space; SIGNED: negated when its normal e0 x e1 (normalised) points
// away from n (minAngleMetricTri(p, n) / maxAngleMetricTri(p, n); without n the unsigned metric)
template <bool MAXA, bool SIGNED>
__device__ __forceinline__ float tri3d_angle(const float* p0, const float* p1, const float* p2, float nx, float ny,
                                             float nz) {
    float u[3], v[3], w[3], e0[3], e1[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        e0[a] = p1[a] - p0[a]; e1[a] = p2[a] - p1[a];
        u[a] = p0[a] - p1[a];   // angle at p1: (p0 - p1, p2 - p1) = (u, e1)
        v[a] = p1[a] - p2[a];   // angle at p2: (p1 - p2, p0 - p2) = (v, w)
        w[a] = p0[a] - p2[a];
    }
    const float m0[3] = { -w[0], -w[1], -w[2] };   // angle at p0: (p2 - p0, p1 - p0) = (-w, e0)
    const float c1 = ang_cos3(u, e1), c2 = ang_cos3(v, w), c3 = ang_cos3(m0, e0);
    float q = angle_q<MAXA>(fmaxf(fmaxf(c1, c2), c3), fminf(fminf(c1, c2), c3));
    if (SIGNED) {
        const float tx = e0[1] * e1[2] - e0[2] * e1[1], ty = e0[2] * e1[0] - e0[0] * e1[2], tz = e0[0] * e1[1] - e0[1] * e1[0];
        const float len = sqrtf((tx * tx + ty * ty) + tz * tz);
        const float nd = ((tx / len) * nx + (ty / len) * ny) + (tz / len) * nz;
        if (nd < 0.f) q = -q;
    }
    return q;
}

// tetrahedron (p0, p1, p2, p3): dihedral angles between the face normals
template <bool MAXA>
__device__ __forceinline__ float tet_angle(const float* p0, const float* p1, const float* p2, const float* p3) {
    float e[6][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        e[0][a] = p1[a] - p0[a]; e[1][a] = p2[a] - p0[a]; e[2][a] = p3[a] - p0[a];
        e[3][a] = p2[a] - p1[a]; e[4][a] = p3[a] - p1[a]; e[5][a] = p3[a] - p2[a];
    }
    auto cross = [](const float* u, const float* v, float* o) {
        o[0] = u[1] * v[2] - u[2] * v[1];
        o[1] = u[2] * v[0] - u[0] * v[2];
        o[2] = u[0] * v[1] - u[1] * v[0];
    };
    float x[3];
    cross(e[1], e[2], x);
    const float vol = (1.f / 6.f) * ((e[0][0] * x[0] + e[0][1] * x[1]) + e[0][2] * x[2]);
    if (vol < 0.f) return vol;
    float n[4][3];
    cross(e[0], e[2], n[0]);
    cross(e[3], e[4], n[1]);
    cross(e[1], e[0], n[2]);
    cross(e[2], e[1], n[3]);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float len = sqrtf((n[i][0] * n[i][0] + n[i][1] * n[i][1]) + n[i][2] * n[i][2]);
        n[i][0] /= len; n[i][1] /= len; n[i][2] /= len;
    }
    float cmax = -FLT_MAX, cmin = FLT_MAX;
    const int P[6][2] = { { 0, 1 }, { 0, 2 }, { 0, 3 }, { 1, 2 }, { 1, 3 }, { 2, 3 } };
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const float* a = n[P[q][0]];
        const float m[3] = { -a[0], -a[1], -a[2] };
        const float c = ang_cos3(m, n[P[q][1]]);
        cmax = fmaxf(cmax, c);
        cmin = fminf(cmin, c);
    }
    return angle_q<MAXA>(cmax, cmin);
}

}  // namespace vsdmo
