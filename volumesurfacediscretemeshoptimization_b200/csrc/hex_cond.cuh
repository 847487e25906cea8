// hex_cond.cuh -- condition-number quality of hexahedra, an addition to the reference's
// criteria (its hex meshes are judged by shapeMetricHex, dmo/DMOQualityHex.h:54-71).
//
// With the corners read in the reference's order P = v4 v5 v6 v7 v0 v1 v2 v3 (bottom face
// P0..P3, top face P4..P7), corner i has the Jacobian A_i of its three edges
//   c0 (P1-P0, P3-P0, P4-P0)  c1 (P2-P1, P0-P1, P5-P1)  c2 (P3-P2, P1-P2, P6-P2)
//   c3 (P0-P3, P2-P3, P7-P3)  c4 (P7-P4, P5-P4, P0-P4)  c5 (P4-P5, P6-P5, P1-P5)
//   c6 (P5-P6, P7-P6, P2-P6)  c7 (P6-P7, P4-P7, P3-P7)
// (right-handed: det A_i = 1 on the unit cube). The corner quality is the inverse condition
// number 1 / kappa(A) = 3 |det A| / (|A|_F |adj A|_F), signed by det A (negative at an
// inverted corner, 0 when an edge set is degenerate); the element quality is its minimum over
// the 8 corners (1 for the unit cube). The searches compare the monotone key
// det |det| / (|A|_F^2 |adj A|_F^2) instead, which needs no square root.
#pragma once
#include <cuda_runtime.h>

namespace vsdmo {

static __host__ __device__ __forceinline__ void hc_cross(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static __host__ __device__ __forceinline__ float hc_dot(const float* a, const float* b) {
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

// det of (e1, e2, e3) and den = |A|_F^2 |adj A|_F^2
static __host__ __device__ __forceinline__ void hc_corner(const float* e1, const float* e2, const float* e3,
                                                          float& det, float& den) {
    float x[3], y[3], z[3];
    hc_cross(e2, e3, x);
    det = hc_dot(e1, x);
    const float F2 = (hc_dot(e1, e1) + hc_dot(e2, e2)) + hc_dot(e3, e3);
    hc_cross(e3, e1, y);
    hc_cross(e1, e2, z);
    const float G2 = (hc_dot(x, x) + hc_dot(y, y)) + hc_dot(z, z);
    den = F2 * G2;
}

// search key of the corner with edges (a - o, b - o, c - o)
static __host__ __device__ __forceinline__ float hc_key(const float* o, const float* a, const float* b, const float* c) {
    const float e1[3] = { a[0] - o[0], a[1] - o[1], a[2] - o[2] };
    const float e2[3] = { b[0] - o[0], b[1] - o[1], b[2] - o[2] };
    const float e3[3] = { c[0] - o[0], c[1] - o[1], c[2] - o[2] };
    float det, den;
    hc_corner(e1, e2, e3, det, den);
    return den > 0.f ? (det * fabsf(det)) / den : 0.f;
}

// quality of the corner with edges (a - o, b - o, c - o)
static __host__ __device__ __forceinline__ float hc_quality(const float* o, const float* a, const float* b,
                                                            const float* c) {
    const float e1[3] = { a[0] - o[0], a[1] - o[1], a[2] - o[2] };
    const float e2[3] = { b[0] - o[0], b[1] - o[1], b[2] - o[2] };
    const float e3[3] = { c[0] - o[0], c[1] - o[1], c[2] - o[2] };
    float det, den;
    hc_corner(e1, e2, e3, det, den);
    return den > 0.f ? (3.f * det) / sqrtf(den) : 0.f;
}

// element quality of the hex with corners v[0..7] in the mesh's order
static __host__ __device__ __forceinline__ float hc_element_quality(const float (*v)[3]) {
    const float* P[8] = { v[4], v[5], v[6], v[7], v[0], v[1], v[2], v[3] };
    float q = hc_quality(P[0], P[1], P[3], P[4]);
    q = fminf(q, hc_quality(P[1], P[2], P[0], P[5]));
    q = fminf(q, hc_quality(P[2], P[3], P[1], P[6]));
    q = fminf(q, hc_quality(P[3], P[0], P[2], P[7]));
    q = fminf(q, hc_quality(P[4], P[7], P[5], P[0]));
    q = fminf(q, hc_quality(P[5], P[4], P[6], P[1]));
    q = fminf(q, hc_quality(P[6], P[5], P[7], P[2]));
    q = fminf(q, hc_quality(P[7], P[6], P[4], P[3]));
    return q;
}

// A halfhex of the vertex: its hex with the vertex p as corner 0 and the other corners
// r[0..6] (corners 1..7), so P4 = p, P5..P7 = r0..r2, P0..P3 = r3..r6. Corners c1, c2, c3 and
// c6 do not touch p: their minimum key is the halfhex's constant part.
static __host__ __device__ __forceinline__ float hc_const_key(const float (*r)[3]) {
    float k = hc_key(r[4], r[5], r[3], r[0]);           // c1
    k = fminf(k, hc_key(r[5], r[6], r[4], r[1]));       // c2
    k = fminf(k, hc_key(r[6], r[3], r[5], r[2]));       // c3
    k = fminf(k, hc_key(r[1], r[0], r[2], r[5]));       // c6
    return k;
}

// the halfhex's key at p: its constant part and the four corners that touch p
static __host__ __device__ __forceinline__ float hc_halfhex_key(const float (*r)[3], float ck, const float* p) {
    float k = fminf(ck, hc_key(p, r[2], r[0], r[3]));   // c4
    k = fminf(k, hc_key(r[3], r[4], r[6], p));          // c0
    k = fminf(k, hc_key(r[0], p, r[1], r[4]));          // c5
    k = fminf(k, hc_key(r[2], r[1], p, r[6]));          // c7
    return k;
}

}  // namespace vsdmo
