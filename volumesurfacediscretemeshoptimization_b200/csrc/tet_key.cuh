// tet_key.cuh -- the tet ring key of the plain search, shared by the interior search
// (dmo_kernels.cu) and the boundary-surface passes of tet meshes (surf_kernels.cu).
//
// Relative to the vertex and scaled by an exact power of two, the determinant of tet (p, a, b, c)
// is affine in the candidate p (det = d0 - n.p) and the sum of its six squared edge lengths
// quadratic (L = C - 2 s.p + 3|p|^2); the mean ratio 12 cbrt(9) cbrt(det^2) / L is compared
// through the monotone transform det^2 / L^3 (a flipped tet keys the ring by its most negative
// det, the analogue of the reference returning the negative volume).
#pragma once
#include <cuda_runtime.h>

namespace vsdmo {

// 2^e as a float when it is a normal number, else 0. Multiplying by it is exactly ldexpf(x, e)
// (both are the correctly rounded value of x 2^e), at the cost of one multiply.
static __device__ __forceinline__ float exp2_exact(int e) { return (e >= -126 && e <= 127) ? __int_as_float((e + 127) << 23) : 0.f; }
static __device__ __forceinline__ float scale2(float x, float p, int e) { return p != 0.f ? x * p : ldexpf(x, e); }

// coefficients of tet (p, a, b, c) in scaled local coordinates
static __device__ __forceinline__ void tet_coeffs(float ax, float ay, float az, float bx, float by, float bz,
                                           float cx, float cy, float cz, float4& K0, float4& K1) {
    float ux = bx - ax, uy = by - ay, uz = bz - az;
    float wx = cx - ax, wy = cy - ay, wz = cz - az;
    float vx = cx - bx, vy = cy - by, vz = cz - bz;
    float nx = uy * wz - uz * wy;
    float ny = uz * wx - ux * wz;
    float nz = ux * wy - uy * wx;
    float d0 = (ax * nx + ay * ny) + az * nz;
    float sx = (ax + bx) + cx, sy = (ay + by) + cy, sz = (az + bz) + cz;
    float a2 = (ax * ax + ay * ay) + az * az;
    float b2 = (bx * bx + by * by) + bz * bz;
    float c2 = (cx * cx + cy * cy) + cz * cz;
    float u2 = (ux * ux + uy * uy) + uz * uz;
    float w2 = (wx * wx + wy * wy) + wz * wz;
    float v2 = (vx * vx + vy * vy) + vz * vz;
    K0 = make_float4(-nx, -ny, -nz, d0);
    K1 = make_float4(-2.0f * sx, -2.0f * sy, -2.0f * sz, ((((a2 + b2) + c2) + u2) + w2) + v2);
}

// key of one candidate (used for the current position)
static __device__ float tet_key1(const float4* co, int k, float x, float y, float z) {
    const float tx = (3.0f * x) * x, ty = (3.0f * y) * y, tz = (3.0f * z) * z;
    float N = 0.f, D = 1.f, dm = 0.f;
    for (int t = 0; t < k; ++t) {
        const float4 c0 = co[2 * t], c1 = co[2 * t + 1];
        float detA = fmaf(c0.x, x, c0.w);
        float LA = c1.w + fmaf(c1.x, x, tx);
        float detB = fmaf(c0.y, y, detA);
        float LB = LA + fmaf(c1.y, y, ty);
        float det = fmaf(c0.z, z, detB);
        float L = LB + fmaf(c1.z, z, tz);
        float num = det * det;
        float den = (L * L) * L;
        if (t == 0) { N = num; D = den; dm = det; continue; }
        if (num * D < N * den) { N = num; D = den; }
        dm = fminf(dm, det);
    }
    return dm < 0.f ? dm : N / D;
}

// tet_key1 at the local origin (the vertex itself): det = d0 and L = C exactly there (every term
// that carries the candidate is a product with +-0 added to them), so the same fold runs on the
// constant coefficients alone and returns the same key
static __device__ float tet_key_origin(const float4* co, int k) {
    float N = 0.f, D = 1.f, dm = 0.f;
    for (int t = 0; t < k; ++t) {
        const float det = co[2 * t].w, L = co[2 * t + 1].w;
        const float num = det * det;
        const float den = (L * L) * L;
        if (t == 0) { N = num; D = den; dm = det; continue; }
        if (num * D < N * den) { N = num; D = den; }
        dm = fminf(dm, det);
    }
    return dm < 0.f ? dm : N / D;
}

}  // namespace vsdmo
