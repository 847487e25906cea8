// quad_cond.cuh -- condition-number quality of quadrilaterals, an addition to the reference's
// criteria (its quads are judged by meanRatioMetricQuad, dmo/DMOQualityQuad.h:13-50).
#pragma once
#include <cuda_runtime.h>

namespace vsdmo {

static __device__ __forceinline__ float qc_dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return (ax * bx + ay * by) + az * bz;
}

// per corner with edges e1, e2 to its neighbours, 2 det / (|e1|^2 + |e2|^2),
// det = (e1 x e2) . n signed by the vertex normal, |e1 x e2| without; 1 at a square corner;
// the quad takes its smallest corner
template <bool SIGNED>
static __device__ __forceinline__ float quad_cond_corner(float ox, float oy, float oz, float ax, float ay, float az, float bx,
                                                  float by, float bz, float3 n) {
    const float e1x = ax - ox, e1y = ay - oy, e1z = az - oz;
    const float e2x = bx - ox, e2y = by - oy, e2z = bz - oz;
    const float cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
    const float F2 = qc_dot3(e1x, e1y, e1z, e1x, e1y, e1z) + qc_dot3(e2x, e2y, e2z, e2x, e2y, e2z);
    const float det = SIGNED ? qc_dot3(cx, cy, cz, n.x, n.y, n.z) : sqrtf(qc_dot3(cx, cy, cz, cx, cy, cz));
    return F2 > 0.f ? (2.f * det) / F2 : 0.f;
}

template <bool SIGNED>
static __device__ __forceinline__ float quad_cond(float p0x, float p0y, float p0z, float4 p1, float4 p2, float4 p3, float3 n) {
    float q = quad_cond_corner<SIGNED>(p0x, p0y, p0z, p1.x, p1.y, p1.z, p3.x, p3.y, p3.z, n);
    q = fminf(q, quad_cond_corner<SIGNED>(p1.x, p1.y, p1.z, p2.x, p2.y, p2.z, p0x, p0y, p0z, n));
    q = fminf(q, quad_cond_corner<SIGNED>(p2.x, p2.y, p2.z, p3.x, p3.y, p3.z, p1.x, p1.y, p1.z, n));
    q = fminf(q, quad_cond_corner<SIGNED>(p3.x, p3.y, p3.z, p0x, p0y, p0z, p2.x, p2.y, p2.z, n));
    return q;
}

}  // namespace vsdmo
