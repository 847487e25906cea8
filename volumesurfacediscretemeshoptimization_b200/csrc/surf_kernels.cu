// surf_kernels.cu -- surface DMO of triangle and quad meshes (free surface vertices).
//
// Per optimiser the state of the reference's DMOTriClass / DMOQuadClass (dmo/DMOTri.cu:80-126,
// dmo/DMOQuad.cu:78-123): the initial positions X0, one local quadric surface per surface
// vertex fitted to them, and for every vertex the nearest initial vertex nn[v] whose surface
// is used for it. Kernels:
//
//   k_surface_fit   computeLocalCoordinates + computeLocalSurface1/2 (dmo/surfaceP/Surface.h:66-93,
//                   Surface.cu:11-104): frame t1 = n x (q0 - p), t2 = n x t1, least squares
//                   quadric w = a u^2 + b uv + c v^2 over the centre and its 1-ring (plus the
//                   midpoint of neighbours 1 and 2 for valence 4; optionally the 2-ring as
//                   well, an addition the reference does not have); the 3x3 normal equations are
//                   solved by LU with partial pivoting in registers (the reference calls the
//                   batched cuBLAS getrf/getrs; the published algorithm is restated here).
//   k_update_nn     k_updateNearestNeighbor (dmo/DMOCommon.cu:11-42): greedy walk over the
//                   initial positions to the initial vertex nearest to the current position.
//   k_dmo_surf<FK,Q> k_optimizeHierarchical2D (dmo/DMOTriImplCub.h:26-201 for FK = 3,
//                   dmo/DMOQuadImplCub.h:24-209 for FK = 4): 8 x 8 grid in the (u, v) frame of
//                   the surface of nn[v], each candidate projected by the inverse-distance blend
//                   over the 1-ring surfaces (localSurfaceEstimationWithFeature,
//                   dmo/SurfaceEstimation.h:122-197), three levels, the normal-signed mean ratio
//                   of the ring (meanRatioMetricTri(p, n), dmo/DMOQualityTri.h:276-293;
//                   meanRatioMetricQuad(p, n), dmo/DMOQualityQuad.h:30-50).
//
// Layout: one warp per vertex. The lanes stage the ring positions, the neighbours' surfaces
// (64 B each) and their nearest initial positions in shared memory; lane t evaluates the
// candidates (i, j) = (t >> 3, t & 7) and (i + 4, j) of the reference's 32-thread block and
// keeps the better one. The winning lane is the first maximum in lane order (a scan of the 32
// values, which is what the reference's cub::BlockReduce ArgMax gives).
//
// Arithmetic: the triangle ring minimum is compared as the fraction sign |n_t|^2 / L^2
// (monotone in the reference's 2 sqrt3 sign |n_t| / L), without its square root and division
// per element; the quad metric is the reference formula. Projections and blends use a fixed
// operation order, reproduced by the oracle's f32 mirror bit for bit (built with
// --fmad=false here and without contraction there).
#include "vsdmo_internal.cuh"
#include "tet_key.cuh"
#include "hex_key.cuh"
#include "angle_metrics.cuh"
#include "quad_cond.cuh"
#include <algorithm>
#include <cfloat>

namespace vsdmo {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int SURF_WARPS = 4;
constexpr int SURF_MAX_RING = 64;
constexpr float SURF_EPS = 1.19209e-07f;   // EPSILON of the reference's surface code
constexpr int SECT_TABLE = 20;              // TABLE_SIZE of dmo/surfaceP/SurfaceCommon.h: halfedges of a feature vertex
constexpr int SECT_LIST = 40;               // MAX_NEIGHBORS: points of one sector
constexpr int TET_SURF_MAX_RING = 256;      // tets of a boundary vertex in the boundary passes
constexpr int HEX_SURF_MAX_RING = 64;       // hexahedra of a boundary vertex in the boundary passes

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return (ax * bx + ay * by) + az * bz;
}

// ---- quadric fit ----------------------------------------------------------------------------
// LU with partial pivoting of a 3 x 3 system (row-major A), solution returned in b
__device__ void solve3(float A[3][3], float b[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int p = k;
#pragma unroll
        for (int i = k + 1; i < 3; ++i) if (fabsf(A[i][k]) > fabsf(A[p][k])) p = i;
        if (p != k) {
#pragma unroll
            for (int j = 0; j < 3; ++j) { float t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t; }
            float t = b[k]; b[k] = b[p]; b[p] = t;
        }
#pragma unroll
        for (int i = k + 1; i < 3; ++i) {
            const float f = A[i][k] / A[k][k];
#pragma unroll
            for (int j = k + 1; j < 3; ++j) A[i][j] = A[i][j] - f * A[k][j];
            b[i] = b[i] - f * b[k];
        }
    }
    b[2] = b[2] / A[2][2];
    b[1] = (b[1] - A[1][2] * b[2]) / A[1][1];
    b[0] = ((b[0] - A[0][1] * b[1]) - A[0][2] * b[2]) / A[0][0];
}

// LS[4v + 0..3] = (p0, a), (t1, b), (t2, c), (n, numPoints)
// ring2 = 1: the fit takes the 2-ring too -- after the 1-ring, the ring vertices of each 1-ring
// vertex in row order, each vertex once (the first occurrence), the vertex itself excluded;
// at most 63 points either way.
__global__ void k_surface_fit(int nS, const int* __restrict__ rowptr, const int4* __restrict__ he,
                              const float4* __restrict__ pos, const float* __restrict__ vn, float4* __restrict__ LS,
                              int ring2) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nS; v += gridDim.x * blockDim.x) {
        const float4 c = pos[v];
        const int b = rowptr[v], k = rowptr[v + 1] - b;
        int ids[62];
        int nb = 0;
        for (int i = 0; i < k && nb < 62; ++i) ids[nb++] = he[b + i].x;   // the reference keeps at most 63 points
        if (ring2) {
            const int n1 = nb;
            for (int i = 0; i < n1 && nb < 62; ++i) {
                const int u = ids[i];
                for (int j = rowptr[u]; j < rowptr[u + 1] && nb < 62; ++j) {
                    const int w = he[j].x;
                    bool seen = w == v;
                    for (int a = 0; a < nb && !seen; ++a) seen = ids[a] == w;
                    if (!seen) ids[nb++] = w;
                }
            }
        }
        const int np = 1 + nb + (1 + nb == 5 ? 1 : 0);
        float n[3] = { vn[3 * v], vn[3 * v + 1], vn[3 * v + 2] };
        const float4 q0 = pos[he[b].x];
        float rv[3] = { q0.x - c.x, q0.y - c.y, q0.z - c.z };
        float cr[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        if (sqrtf(dot3(cr[0], cr[1], cr[2], cr[0], cr[1], cr[2])) < 10.f * SURF_EPS) {
            rv[0] = n[0]; rv[1] = n[2]; rv[2] = -n[1];
        }
        float t1[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        float t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
        const float ln = sqrtf(dot3(n[0], n[1], n[2], n[0], n[1], n[2]));
        const float l1 = sqrtf(dot3(t1[0], t1[1], t1[2], t1[0], t1[1], t1[2]));
        const float l2 = sqrtf(dot3(t2[0], t2[1], t2[2], t2[0], t2[1], t2[2]));
#pragma unroll
        for (int a = 0; a < 3; ++a) { n[a] = n[a] / ln; t1[a] = t1[a] / l1; t2[a] = t2[a] / l2; }
        float M00 = 0.f, M01 = 0.f, M11 = 0.f, M12 = 0.f, M22 = 0.f, r0 = 0.f, r1 = 0.f, r2 = 0.f;
        for (int i = 0; i < np; ++i) {
            float px, py, pz;
            if (i == 0) {
                px = c.x; py = c.y; pz = c.z;
            } else if (i <= nb) {
                const float4 q = pos[ids[i - 1]];
                px = q.x; py = q.y; pz = q.z;
            } else {  // valence 4: midpoint of points 2 and 3 (neighbours 1 and 2)
                const float4 qa = pos[ids[1]], qb = pos[ids[2]];
                px = 0.5f * (qa.x + qb.x); py = 0.5f * (qa.y + qb.y); pz = 0.5f * (qa.z + qb.z);
            }
            const float dx = px - c.x, dy = py - c.y, dz = pz - c.z;
            const float u = dot3(t1[0], t1[1], t1[2], dx, dy, dz);
            const float w2 = dot3(t2[0], t2[1], t2[2], dx, dy, dz);
            const float w = dot3(n[0], n[1], n[2], dx, dy, dz);
            const float uu = u * u, uv = u * w2, v2 = w2 * w2;
            r0 = r0 + uu * w; r1 = r1 + uv * w; r2 = r2 + v2 * w;
            M00 = M00 + uu * uu; M01 = M01 + uu * uv; M11 = M11 + uu * v2; M12 = M12 + uv * v2; M22 = M22 + v2 * v2;
        }
        float A[3][3] = { { M00, M01, M11 }, { M01, M11, M12 }, { M11, M12, M22 } };
        float s[3] = { r0, r1, r2 };
        solve3(A, s);
        if (np <= 4) { s[0] = 0.f; s[1] = 0.f; s[2] = 0.f; }
#pragma unroll
        for (int a = 0; a < 3; ++a) if (s[a] != s[a]) s[a] = 0.f;
        LS[4L * v + 0] = make_float4(c.x, c.y, c.z, s[0]);
        LS[4L * v + 1] = make_float4(t1[0], t1[1], t1[2], s[1]);
        LS[4L * v + 2] = make_float4(t2[0], t2[1], t2[2], s[2]);
        LS[4L * v + 3] = make_float4(n[0], n[1], n[2], (float)np);
    }
}

// ---- nearest initial vertex -------------------------------------------------------------------
__global__ void k_update_nn(int nS, int nFree, const int* __restrict__ rowptr, const int4* __restrict__ he,
                            const float4* __restrict__ pos, const float4* __restrict__ X0, int* __restrict__ nn) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nS; v += gridDim.x * blockDim.x) {
        const float4 p = pos[v];
        int vh = nn[v];
        const float4 pi = X0[vh];
        float sd = dot3(p.x - pi.x, p.y - pi.y, p.z - pi.z, p.x - pi.x, p.y - pi.y, p.z - pi.z);
        const bool fv = v >= nFree;
        int vnew;
        // every step strictly lowers the distance, so the walk visits at most nS vertices
        int steps = 0;
        do {
            vnew = vh;
            for (int i = rowptr[vnew]; i < rowptr[vnew + 1]; ++i) {
                const int d = he[i].x;
                if (fv != (d >= nFree)) continue;
                const float4 q = X0[d];
                const float ex = p.x - q.x, ey = p.y - q.y, ez = p.z - q.z;
                const float s2 = dot3(ex, ey, ez, ex, ey, ez);
                if (s2 < sd) { sd = s2; vh = d; }
            }
        } while (vnew != vh && ++steps <= nS);
        nn[v] = vnew;
    }
}

// ---- grid search --------------------------------------------------------------------------------
struct Surf {
    float4 l0, l1, l2, l3;   // (p0, a), (t1, b), (t2, c), (n, numPoints)
};

__device__ __forceinline__ float poly(const float4& l0, const float4& l1, const float4& l2, float u, float v) {
    return (((l0.w * u) * u) + ((l1.w * u) * v)) + ((l2.w * v) * v);
}

// blended projection of (u, v) of the vertex's own surface onto the ring's surfaces
__device__ __forceinline__ float3 estimate(const Surf& L, const float4 x0, const float4* __restrict__ nbL,
                                           const float4* __restrict__ nbX, int k, float u, float v) {
    const float w = poly(L.l0, L.l1, L.l2, u, v);
    const float pwx = ((L.l0.x + u * L.l1.x) + v * L.l2.x) + w * L.l3.x;
    const float pwy = ((L.l0.y + u * L.l1.y) + v * L.l2.y) + w * L.l3.y;
    const float pwz = ((L.l0.z + u * L.l1.z) + v * L.l2.z) + w * L.l3.z;
    const float dx = x0.x - pwx, dy = x0.y - pwy, dz = x0.z - pwz;
    const float id = 1.0f / (dot3(dx, dy, dz, dx, dy, dz) + SURF_EPS);
    float isum = id;
    float ax = pwx * id, ay = pwy * id, az = pwz * id;
    for (int i = 0; i < k; ++i) {
        const float4 xn = nbX[i];
        const float ex = xn.x - pwx, ey = xn.y - pwy, ez = xn.z - pwz;
        const float idn = 1.0f / (dot3(ex, ey, ez, ex, ey, ez) + SURF_EPS);
        isum = isum + idn;
        const float4 m0 = nbL[4 * i], m1 = nbL[4 * i + 1], m2 = nbL[4 * i + 2], m3 = nbL[4 * i + 3];
        const float qx = pwx - m0.x, qy = pwy - m0.y, qz = pwz - m0.z;
        const float lu = dot3(qx, qy, qz, m1.x, m1.y, m1.z);
        const float lv = dot3(qx, qy, qz, m2.x, m2.y, m2.z);
        const float lw = poly(m0, m1, m2, lu, lv);
        const float p2x = ((m0.x + lu * m1.x) + lv * m2.x) + lw * m3.x;
        const float p2y = ((m0.y + lu * m1.y) + lv * m2.y) + lw * m3.y;
        const float p2z = ((m0.z + lu * m1.z) + lv * m2.z) + lw * m3.z;
        ax = ax + p2x * idn; ay = ay + p2y * idn; az = az + p2z * idn;
    }
    const float inv = 1.0f / isum;
    return make_float3(ax * inv, ay * inv, az * inv);
}

// ring key of a triangle fan: min over the fan of sign(n_t . n) |n_t|^2 / L^2 (unsigned without n)
template <bool SIGNED>
__device__ __forceinline__ float ring_key_tri(const float4* __restrict__ ring, int k, float px, float py, float pz,
                                              float3 n) {
    float N = 0.f, D = 1.f;
    for (int i = 0; i < k; ++i) {
        const float4 a = ring[i], b = ring[i + 1];
        const float e0x = a.x - px, e0y = a.y - py, e0z = a.z - pz;
        const float e1x = b.x - px, e1y = b.y - py, e1z = b.z - pz;
        const float e2x = b.x - a.x, e2y = b.y - a.y, e2z = b.z - a.z;
        const float l = (dot3(e0x, e0y, e0z, e0x, e0y, e0z) + dot3(e1x, e1y, e1z, e1x, e1y, e1z)) +
                        dot3(e2x, e2y, e2z, e2x, e2y, e2z);
        const float nx = e0y * e1z - e0z * e1y, ny = e0z * e1x - e0x * e1z, nz = e0x * e1y - e0y * e1x;
        const float a2 = dot3(nx, ny, nz, nx, ny, nz);
        float num = a2;
        if (SIGNED) {
            const float dn = dot3(nx, ny, nz, n.x, n.y, n.z);
            num = dn > 0.f ? a2 : (dn < 0.f ? -a2 : 0.f);
        }
        const float den = l * l;
        if (i == 0) { N = num; D = den; continue; }
        if (num * D < N * den) { N = num; D = den; }
    }
    return N / D;
}

// meanRatioMetricQuad(p, n) / (p): 2 (A1 + A2) / sum |e|^2, -1 when a corner normal leaves n
template <bool SIGNED>
__device__ __forceinline__ float quad_metric(float p0x, float p0y, float p0z, float4 p1, float4 p2, float4 p3, float3 n) {
    const float e0x = p1.x - p0x, e0y = p1.y - p0y, e0z = p1.z - p0z;
    const float e1x = p2.x - p1.x, e1y = p2.y - p1.y, e1z = p2.z - p1.z;
    const float e2x = p3.x - p2.x, e2y = p3.y - p2.y, e2z = p3.z - p2.z;
    const float e3x = p0x - p3.x, e3y = p0y - p3.y, e3z = p0z - p3.z;
    const float l = ((dot3(e0x, e0y, e0z, e0x, e0y, e0z) + dot3(e1x, e1y, e1z, e1x, e1y, e1z)) +
                     dot3(e2x, e2y, e2z, e2x, e2y, e2z)) + dot3(e3x, e3y, e3z, e3x, e3y, e3z);
    const float m0x = -e0x, m0y = -e0y, m0z = -e0z, m2x = -e2x, m2y = -e2y, m2z = -e2z;
    const float c1x = e1y * m0z - e1z * m0y, c1y = e1z * m0x - e1x * m0z, c1z = e1x * m0y - e1y * m0x;
    const float c2x = e3y * m2z - e3z * m2y, c2y = e3z * m2x - e3x * m2z, c2z = e3x * m2y - e3y * m2x;
    const float a1 = sqrtf(dot3(c1x, c1y, c1z, c1x, c1y, c1z));
    const float a2 = sqrtf(dot3(c2x, c2y, c2z, c2x, c2y, c2z));
    if (SIGNED) {
        const float d1 = dot3(c1x, c1y, c1z, n.x, n.y, n.z) / a1;
        const float d2 = dot3(c2x, c2y, c2z, n.x, n.y, n.z) / a2;
        if (d1 < 0.7f || d2 < 0.7f) return -1.f;
    }
    return (2.f * (a1 + a2)) / l;
}

template <bool SIGNED>
__device__ __forceinline__ float ring_key_quad_cond(const float4* __restrict__ ring, int k, float px, float py,
                                                    float pz, float3 n) {
    float q = 0.f;
    for (int i = 0; i < k; ++i) {
        const float v = quad_cond<SIGNED>(px, py, pz, ring[2 * i], ring[2 * i + 1], ring[2 * i + 2], n);
        q = i == 0 ? v : fminf(q, v);
    }
    return q;
}

template <bool SIGNED>
__device__ __forceinline__ float ring_key_quad(const float4* __restrict__ ring, int k, float px, float py, float pz,
                                               float3 n) {
    float q = 0.f;
    for (int i = 0; i < k; ++i) {
        const float v = quad_metric<SIGNED>(px, py, pz, ring[2 * i], ring[2 * i + 1], ring[2 * i + 2], n);
        q = i == 0 ? v : fminf(q, v);
    }
    return q;
}

// angle criteria on a triangle fan: min over the fan of minAngleMetricTri / maxAngleMetricTri
// of (p, ring[i], ring[i + 1]) (qualityShapeMinAMTri / MaxAMTri, dmo/DMOQualityTri.h:89-121,
// 205-237), signed by n when SIGNED
template <bool MAXA, bool SIGNED>
__device__ __forceinline__ float ring_angle_tri(const float4* __restrict__ ring, int k, float px, float py, float pz,
                                                float3 n) {
    const float p[3] = { px, py, pz };
    float q = FLT_MAX;
    for (int i = 0; i < k; ++i) {
        const float4 a = ring[i], b = ring[i + 1];
        const float pa[3] = { a.x, a.y, a.z }, pb[3] = { b.x, b.y, b.z };
        q = fminf(q, tri3d_angle<MAXA, SIGNED>(p, pa, pb, n.x, n.y, n.z));
    }
    return q;
}

// ring quality of a surface vertex; Q: 0 mean ratio, 1 min angle, 2 max angle (triangles),
// 3 condition number (quads)
template <int FK, bool SIGNED, int Q = 0>
__device__ __forceinline__ float ring_key(const float4* ring, int k, float px, float py, float pz, float3 n) {
    if (FK == 3 && Q == 1) return ring_angle_tri<false, SIGNED>(ring, k, px, py, pz, n);
    if (FK == 3 && Q == 2) return ring_angle_tri<true, SIGNED>(ring, k, px, py, pz, n);
    if (FK == 3) return ring_key_tri<SIGNED>(ring, k, px, py, pz, n);
    if (Q == 3) return ring_key_quad_cond<SIGNED>(ring, k, px, py, pz, n);
    return ring_key_quad<SIGNED>(ring, k, px, py, pz, n);
}

// shared memory per warp, in float4: ring [2 maxk + 1], neighbour surfaces [4 maxk], X0 [maxk]
__host__ __device__ constexpr int surf_warp_f4(int maxk) { return 7 * maxk + 1; }

// surface of ring neighbour vN for vertex v: its nearest initial vertex's surface, or for a feature
// nearest initial vertex the sector surface of its halfedge whose target is nearest to v
// (positions Xs taken at the start of the colour class)
__device__ __forceinline__ const float4* neighbour_surface(int v, int nnN, const float4* __restrict__ LS,
                                                           const int* __restrict__ rowptr, const int4* __restrict__ he,
                                                           const int* __restrict__ srow, const int* __restrict__ stab,
                                                           const float4* __restrict__ FS, const float4* __restrict__ Xs,
                                                           int nFree) {
    if (!FS || nnN < nFree) return LS + 4L * nnN;
    const float4 pv = Xs[v];
    float best = FLT_MAX;
    int arg = 0;
    for (int j = rowptr[nnN], idx = 0; j < rowptr[nnN + 1]; ++j, ++idx) {
        const float4 t = Xs[he[j].x];
        const float ex = t.x - pv.x, ey = t.y - pv.y, ez = t.z - pv.z;
        const float d2 = dot3(ex, ey, ez, ex, ey, ez);
        if (d2 < best) { best = d2; arg = idx; }
    }
    return FS + 4L * (srow[nnN - nFree] + stab[SECT_TABLE * (nnN - nFree) + arg]);
}

// Volume rings of a boundary vertex for the boundary passes of volume meshes. stage() reads
// the vertex's ring from pos, scales it by 2^-ex like the interior search (ex from the largest
// per-axis ring distance) and writes its coefficients to co; key(p) is the ring key at the
// absolute position p; md is the grid extent of the reference kernel. stage() returns false
// for a degenerate ring.
struct TetRing {
    // k_optimizeHierarchical2DTet / 1DTet: extent = largest distance to a ring point
    // (dmo/DMOTetImplCub.h:246, 455); 2 float4 of coefficients per tet (tet_key.cuh)
    static constexpr int F4 = 2;
    const float4* co;
    int k, ex;
    float pinv, md;
    float4 c0;
    __device__ bool stage(const float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hf,
                          int v, float4 c, int lane, float4* buf) {
        c0 = c;
        co = buf;
        const int b = rowptr[v];
        k = rowptr[v + 1] - b;
        float mm = 0.f, me = -FLT_MAX;
        for (int t = lane; t < k; t += 32) {
            const int4 h = hf[b + t];
            const int ids[3] = { h.x, h.y, h.z };
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float4 q = pos[ids[j]];
                const float dx = q.x - c0.x, dy = q.y - c0.y, dz = q.z - c0.z;
                mm = fmaxf(mm, fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))));
                me = fmaxf(me, sqrtf(dot3(dx, dy, dz, dx, dy, dz)));
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            mm = fmaxf(mm, __shfl_xor_sync(FULL, mm, o));
            me = fmaxf(me, __shfl_xor_sync(FULL, me, o));
        }
        md = me;
        if (!(mm > 0.f) || !(mm < FLT_MAX)) return false;
        (void)frexpf(mm, &ex);
        pinv = exp2_exact(-ex);
        for (int t = lane; t < k; t += 32) {
            const int4 h = hf[b + t];
            const float4 pa = pos[h.x], pb = pos[h.y], pc = pos[h.z];
            float4 K0, K1;
            tet_coeffs(scale2(pa.x - c0.x, pinv, -ex), scale2(pa.y - c0.y, pinv, -ex), scale2(pa.z - c0.z, pinv, -ex),
                       scale2(pb.x - c0.x, pinv, -ex), scale2(pb.y - c0.y, pinv, -ex), scale2(pb.z - c0.z, pinv, -ex),
                       scale2(pc.x - c0.x, pinv, -ex), scale2(pc.y - c0.y, pinv, -ex), scale2(pc.z - c0.z, pinv, -ex),
                       K0, K1);
            buf[2 * t] = K0;
            buf[2 * t + 1] = K1;
        }
        __syncwarp();
        return true;
    }
    __device__ float key(float px, float py, float pz) const {
        return tet_key1(co, k, scale2(px - c0.x, pinv, -ex), scale2(py - c0.y, pinv, -ex), scale2(pz - c0.z, pinv, -ex));
    }
};

struct HexRing {
    // k_optimizeHierarchical2DHex / 1DHex: extent = smallest distance to a ring point
    // (dmo/DMOHexImplCub.h:246, 448); 43 floats of coefficients per halfhex (hex_key.cuh)
    static constexpr int F4 = HEX_CO / 4;
    const float* co;
    int k, ex;
    float pinv, md, es, ea;
    float4 c0;
    __device__ bool stage(const float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hh,
                          int v, float4 c, int lane, float4* buf) {
        c0 = c;
        float* cf = reinterpret_cast<float*>(buf);
        co = cf;
        const int b = rowptr[v];
        k = rowptr[v + 1] - b;
        float mm = 0.f, me = FLT_MAX;
        for (int idx = lane; idx < 7 * k; idx += 32) {
            const int h = idx / 7, c7 = idx % 7;
            const int4 q = hh[2 * (b + h) + (c7 >> 2)];
            const int cc = c7 & 3;
            const float4 p = pos[cc == 0 ? q.x : (cc == 1 ? q.y : (cc == 2 ? q.z : q.w))];
            const float dx = p.x - c0.x, dy = p.y - c0.y, dz = p.z - c0.z;
            mm = fmaxf(mm, fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))));
            me = fminf(me, sqrtf(dot3(dx, dy, dz, dx, dy, dz)));
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            mm = fmaxf(mm, __shfl_xor_sync(FULL, mm, o));
            me = fminf(me, __shfl_xor_sync(FULL, me, o));
        }
        md = me;
        if (!(mm > 0.f) || !(mm < FLT_MAX)) return false;
        (void)frexpf(mm, &ex);
        pinv = exp2_exact(-ex);
        es = ldexpf(HEX_EPS, -3 * ex);
        ea = ldexpf(HEX_EPS, -2 * ex);
        for (int h = lane; h < k; h += 32) {
            const int4 qa = hh[2 * (b + h)], qb = hh[2 * (b + h) + 1];
            const int us[7] = { qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z };
            float r[7][3];
#pragma unroll
            for (int c7 = 0; c7 < 7; ++c7) {
                const float4 p = pos[us[c7]];
                r[c7][0] = scale2(p.x - c0.x, pinv, -ex);
                r[c7][1] = scale2(p.y - c0.y, pinv, -ex);
                r[c7][2] = scale2(p.z - c0.z, pinv, -ex);
            }
            hex_coeffs(r, es, ea, cf + HEX_CO * h);
        }
        __syncwarp();
        return true;
    }
    __device__ float key(float px, float py, float pz) const {
        return hex_key1(co, k, scale2(px - c0.x, pinv, -ex), scale2(py - c0.y, pinv, -ex), scale2(pz - c0.z, pinv, -ex),
                        es, ea);
    }
};

template <bool MAXA>
struct TetAngleRing {
    // angle criteria on the ring of tets (qualityTetRing with MIN_ANGLE / MAX_ANGLE,
    // dmo/DMOQualityTet.h:165-177): the literal metric per tet (angle_metrics.cuh) on positions
    // relative to the vertex; extent as TetRing
    static constexpr int F4 = 3;
    const float4* r;
    int k;
    float md;
    float4 c0;
    __device__ bool stage(const float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hf,
                          int v, float4 c, int lane, float4* buf) {
        c0 = c;
        r = buf;
        const int b = rowptr[v];
        k = rowptr[v + 1] - b;
        float mm = 0.f, me = -FLT_MAX;
        for (int t = lane; t < k; t += 32) {
            const int4 h = hf[b + t];
            const int ids[3] = { h.x, h.y, h.z };
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float4 q = pos[ids[j]];
                const float dx = q.x - c0.x, dy = q.y - c0.y, dz = q.z - c0.z;
                mm = fmaxf(mm, fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))));
                me = fmaxf(me, sqrtf(dot3(dx, dy, dz, dx, dy, dz)));
                buf[3 * t + j] = make_float4(dx, dy, dz, 0.f);
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            mm = fmaxf(mm, __shfl_xor_sync(FULL, mm, o));
            me = fmaxf(me, __shfl_xor_sync(FULL, me, o));
        }
        md = me;
        __syncwarp();
        return mm > 0.f && mm < FLT_MAX;
    }
    __device__ float key(float px, float py, float pz) const {
        const float p[3] = { px - c0.x, py - c0.y, pz - c0.z };
        float q = FLT_MAX;
        for (int t = 0; t < k; ++t) {
            const float4 a = r[3 * t], b = r[3 * t + 1], c = r[3 * t + 2];
            const float pa[3] = { a.x, a.y, a.z }, pb[3] = { b.x, b.y, b.z }, pc[3] = { c.x, c.y, c.z };
            q = fminf(q, tet_angle<MAXA>(p, pa, pb, pc));
        }
        return q;
    }
};

template <int FK, int Q>
__global__ void __launch_bounds__(SURF_WARPS * 32)
k_dmo_surf(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he,
           const float4* __restrict__ X0, const float4* __restrict__ LS, const int* __restrict__ nn,
           const float* __restrict__ vn, int v0, int v1, float grid_scale, int depth, int maxk,
           const int* __restrict__ srow, const int* __restrict__ stab, const float4* __restrict__ FS,
           const float4* __restrict__ Xs, int nFree) {
    extern __shared__ float4 smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int v = v0 + blockIdx.x * SURF_WARPS + warp;
    if (v >= v1) return;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;   // maxk is the mesh's largest row, checked on the host
    float4* ring = smem + (size_t)warp * surf_warp_f4(maxk);
    float4* nbL = ring + 2 * maxk + 1;
    float4* nbX = nbL + 4 * maxk;
    const float4 c0 = pos[v];
    float md = 0.f;
    for (int i = lane; i < k; i += 32) {
        const int4 h = he[b + i];
        const float4 t = pos[h.x];
        float dx = t.x - c0.x, dy = t.y - c0.y, dz = t.z - c0.z;
        md = fmaxf(md, sqrtf(dot3(dx, dy, dz, dx, dy, dz)));
        if (FK == 3) {
            ring[i] = t;
        } else {
            const float4 t2 = pos[he[h.w].x];
            ring[2 * i] = t;
            ring[2 * i + 1] = t2;
            dx = t2.x - c0.x; dy = t2.y - c0.y; dz = t2.z - c0.z;
            md = fmaxf(md, sqrtf(dot3(dx, dy, dz, dx, dy, dz)));
        }
        const int nnN = nn[h.x];
        const float4* Ls = neighbour_surface(v, nnN, LS, rowptr, he, srow, stab, FS, Xs, nFree);
        nbL[4 * i] = Ls[0];
        nbL[4 * i + 1] = Ls[1];
        nbL[4 * i + 2] = Ls[2];
        nbL[4 * i + 3] = Ls[3];
        nbX[i] = X0[nnN];
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) md = fmaxf(md, __shfl_xor_sync(FULL, md, o));
    __syncwarp();
    if (lane == 0) ring[FK == 3 ? k : 2 * k] = ring[0];
    __syncwarp();

    const int nnv = nn[v];
    Surf L;
    L.l0 = LS[4L * nnv]; L.l1 = LS[4L * nnv + 1]; L.l2 = LS[4L * nnv + 2]; L.l3 = LS[4L * nnv + 3];
    const float4 x0 = X0[nnv];
    const float3 n = make_float3(vn[3L * nnv], vn[3L * nnv + 1], vn[3L * nnv + 2]);
    float cu, cv;
    {
        const float dx = c0.x - L.l0.x, dy = c0.y - L.l0.y, dz = c0.z - L.l0.z;
        cu = dot3(dx, dy, dz, L.l1.x, L.l1.y, L.l1.z);
        cv = dot3(dx, dy, dz, L.l2.x, L.l2.y, L.l2.z);
    }
    float qLast = ring_key<FK, true, Q>(ring, k, c0.x, c0.y, c0.z, n);
    const float qOld = ring_key<FK, false, Q>(ring, k, c0.x, c0.y, c0.z, n);

    const int i1 = lane >> 3, j1 = lane & 7, i2 = i1 + 4;
    const float o1 = (float)(7 - 2 * i1) / 7.f, oj = (float)(7 - 2 * j1) / 7.f, o2 = (float)(7 - 2 * i2) / 7.f;
    float cx = c0.x, cy = c0.y, cz = c0.z;
    float ds = grid_scale, lastMax = -FLT_MAX;
    for (int d = 0; d < depth; ++d) {
        const float S = ds * md;
        const float u1 = fmaf(o1, S, cu), vv = fmaf(oj, S, cv), u2 = fmaf(o2, S, cu);
        const float3 p1 = estimate(L, x0, nbL, nbX, k, u1, vv);
        const float3 p2 = estimate(L, x0, nbL, nbX, k, u2, vv);
        const float q1 = ring_key<FK, true, Q>(ring, k, p1.x, p1.y, p1.z, n);
        const float q2 = ring_key<FK, true, Q>(ring, k, p2.x, p2.y, p2.z, n);
        const bool second = q2 > q1;
        const float val = second ? q2 : q1;
        float bv = __shfl_sync(FULL, val, 0);
        int bt = 0;
        for (int t = 1; t < 32; ++t) {
            const float vt = __shfl_sync(FULL, val, t);
            if (vt > bv) { bv = vt; bt = t; }
        }
        const float bu = __shfl_sync(FULL, second ? u2 : u1, bt);
        const float bw = __shfl_sync(FULL, vv, bt);
        const float bx = __shfl_sync(FULL, second ? p2.x : p1.x, bt);
        const float by = __shfl_sync(FULL, second ? p2.y : p1.y, bt);
        const float bz = __shfl_sync(FULL, second ? p2.z : p1.z, bt);
        if (qLast < bv) { cx = bx; cy = by; cz = bz; cu = bu; cv = bw; qLast = bv; }
        lastMax = bv;
        ds = ds * (2.0f / 7.0f);
    }
    if (lane == 0 && qOld < lastMax) pos[v] = make_float4(cx, cy, cz, c0.w);
}

// ---- feature vertices ---------------------------------------------------------------------------
// fdeg[v]: feature vertices in the ring of surface vertex v; opt[v]: the 1D pass moves feature
// vertex v (two feature ring vertices at >= 160 degrees; k_calcOptFeatureVec, dmo/DMOCommon.h:130-180)
__global__ void k_feature_flags(int nS, int nFree, const int* __restrict__ rowptr, const int4* __restrict__ he,
                                const float4* __restrict__ pos, int* __restrict__ fdeg, uint8_t* __restrict__ opt) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nS; v += gridDim.x * blockDim.x) {
        int cnt = 0, a = -1, b = -1;
        for (int i = rowptr[v]; i < rowptr[v + 1]; ++i) {
            const int d = he[i].x;
            if (d >= nFree) {
                if (cnt == 0) a = d; else if (cnt == 1) b = d;
                ++cnt;
            }
        }
        fdeg[v] = cnt;
        uint8_t o = 0;
        if (v >= nFree && cnt == 2) {
            const float4 p0 = pos[v], pa = pos[a], pb = pos[b];
            const float ux = pa.x - p0.x, uy = pa.y - p0.y, uz = pa.z - p0.z;
            const float wx = pb.x - p0.x, wy = pb.y - p0.y, wz = pb.z - p0.z;
            const float dt = dot3(ux, uy, uz, wx, wy, wz);
            const float len = sqrtf(dot3(ux, uy, uz, ux, uy, uz) * dot3(wx, wy, wz, wx, wy, wz));
            // a float angle, as the reference keeps it (DMOCommon.h:157-158)
            const float ang = (float)(180.0 / 3.14159265358979323846 * (double)acosf(dt / len));
            o = ang >= 160.f ? 1 : 0;
        }
        opt[v] = o;
    }
}

// computeLocalSurface1d (dmo/Surface1D.cu:8-82): curve v = a u^2 in the frame (t2, n), t2 = n x (n x r)
// with r towards the last feature ring vertex; LS1[3v] = (p0, a), (t2, 0), (n, 0)
__global__ void k_surface_fit_1d(int nS, int nFree, int flat, const int* __restrict__ rowptr,
                                 const int4* __restrict__ he, const float4* __restrict__ pos,
                                 const float* __restrict__ vn, float4* __restrict__ LS1) {
    for (int v = nFree + blockIdx.x * blockDim.x + threadIdx.x; v < nS; v += gridDim.x * blockDim.x) {
        int last = -1;
        for (int i = rowptr[v]; i < rowptr[v + 1]; ++i) if (he[i].x >= nFree) last = he[i].x;
        if (last < 0) {
            LS1[3L * v] = make_float4(0.f, 0.f, 0.f, 0.f);
            LS1[3L * v + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
            LS1[3L * v + 2] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const float4 c = pos[v];
        float n[3] = { 0.f, 0.f, 1.f };
        if (!flat) { n[0] = vn[3L * v]; n[1] = vn[3L * v + 1]; n[2] = vn[3L * v + 2]; }
        const float4 q = pos[last];
        float r[3] = { q.x - c.x, q.y - c.y, q.z - c.z };
        const float cr[3] = { n[1] * r[2] - n[2] * r[1], n[2] * r[0] - n[0] * r[2], n[0] * r[1] - n[1] * r[0] };
        if (sqrtf(dot3(cr[0], cr[1], cr[2], cr[0], cr[1], cr[2])) < 10.f * SURF_EPS) { r[0] = n[0]; r[1] = n[2]; r[2] = -n[1]; }
        float t1[3] = { n[1] * r[2] - n[2] * r[1], n[2] * r[0] - n[0] * r[2], n[0] * r[1] - n[1] * r[0] };
        float t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
        const float ln = sqrtf(dot3(n[0], n[1], n[2], n[0], n[1], n[2]));
        const float l1 = sqrtf(dot3(t1[0], t1[1], t1[2], t1[0], t1[1], t1[2]));
        const float l2 = sqrtf(dot3(t2[0], t2[1], t2[2], t2[0], t2[1], t2[2]));
#pragma unroll
        for (int a = 0; a < 3; ++a) { n[a] = n[a] / ln; t1[a] = t1[a] / l1; t2[a] = t2[a] / l2; }
        float ATA = 0.f, ATb = 0.f;
        for (int i = rowptr[v]; i < rowptr[v + 1]; ++i) {
            const int d = he[i].x;
            if (d < nFree) continue;
            const float4 pp = pos[d];
            const float px = pp.x - c.x, py = pp.y - c.y, pz = pp.z - c.z;
            const float u = dot3(t2[0], t2[1], t2[2], px, py, pz), w = dot3(n[0], n[1], n[2], px, py, pz);
            ATb += (u * u) * w;
            ATA += ((u * u) * u) * u;
        }
        LS1[3L * v] = make_float4(c.x, c.y, c.z, ATb / ATA);
        LS1[3L * v + 1] = make_float4(t2[0], t2[1], t2[2], 0.f);
        LS1[3L * v + 2] = make_float4(n[0], n[1], n[2], 0.f);
    }
}

// sectors of a feature vertex (SurfaceFeature.cu:12-85): split of its fan at the feature ring
// vertices; count per feature vertex (plus one closing sector when it is not on a boundary)
__global__ void k_sector_count(int nFeat, int nFree, const int* __restrict__ rowptr, const int4* __restrict__ he,
                               const uint8_t* __restrict__ isB1, int* __restrict__ cnt, int* __restrict__ err) {
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nFeat; idx += gridDim.x * blockDim.x) {
        const int vid = nFree + idx, b = rowptr[vid], e = rowptr[vid + 1];
        if (e - b > SECT_TABLE) { atomicExch(err, 1); cnt[idx] = 0; continue; }
        int sid = 0;
        for (int i = b + 1; i < e; ++i) if (he[i].x >= nFree) ++sid;
        if (!isB1[vid]) ++sid;
        cnt[idx] = sid;
    }
}

// one sector's quadric (computeLocalSurfacesFeature1/2, SurfaceFeature.cu:134-221): the frame of
// the face of the sector's first edge, least squares over the sector's points (+ the midpoint of
// points 2 and 3 when it has 5)
__device__ void sector_fit(const int* L, int np, const int* __restrict__ rowptr, const int4* __restrict__ he,
                           const float4* __restrict__ pos, const float* __restrict__ fn, float4* out) {
    const int vid = L[0];
    const float4 c = pos[vid];
    float P[SECT_LIST + 1][3];
    for (int i = 0; i < np; ++i) { const float4 q = pos[L[i]]; P[i][0] = q.x; P[i][1] = q.y; P[i][2] = q.z; }
    if (np == 5) {
        for (int a = 0; a < 3; ++a) P[5][a] = 0.5f * (P[2][a] + P[3][a]);
        np = 6;
    }
    int f = -1;
    for (int i = rowptr[vid]; i < rowptr[vid + 1]; ++i) if (he[i].x == L[1]) f = he[i].z;
    float n[3] = { fn[3L * f], fn[3L * f + 1], fn[3L * f + 2] };
    const float4 q0 = pos[L[1]];
    float rv[3] = { q0.x - c.x, q0.y - c.y, q0.z - c.z };
    const float cr[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
    if (sqrtf(dot3(cr[0], cr[1], cr[2], cr[0], cr[1], cr[2])) < 10.f * SURF_EPS) { rv[0] = n[0]; rv[1] = n[2]; rv[2] = -n[1]; }
    float t1[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
    float t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
    const float ln = sqrtf(dot3(n[0], n[1], n[2], n[0], n[1], n[2]));
    const float l1 = sqrtf(dot3(t1[0], t1[1], t1[2], t1[0], t1[1], t1[2]));
    const float l2 = sqrtf(dot3(t2[0], t2[1], t2[2], t2[0], t2[1], t2[2]));
    for (int a = 0; a < 3; ++a) { n[a] = n[a] / ln; t1[a] = t1[a] / l1; t2[a] = t2[a] / l2; }
    float M00 = 0.f, M01 = 0.f, M11 = 0.f, M12 = 0.f, M22 = 0.f, r0 = 0.f, r1 = 0.f, r2 = 0.f;
    for (int i = 0; i < np; ++i) {
        const float px = P[i][0] - c.x, py = P[i][1] - c.y, pz = P[i][2] - c.z;
        const float u = dot3(t1[0], t1[1], t1[2], px, py, pz);
        const float vv = dot3(t2[0], t2[1], t2[2], px, py, pz);
        const float w = dot3(n[0], n[1], n[2], px, py, pz);
        const float uu = u * u, uv = u * vv, v2 = vv * vv;
        r0 = r0 + uu * w; r1 = r1 + uv * w; r2 = r2 + v2 * w;
        M00 = M00 + uu * uu; M01 = M01 + uu * uv; M11 = M11 + uu * v2; M12 = M12 + uv * v2; M22 = M22 + v2 * v2;
    }
    float A[3][3] = { { M00, M01, M11 }, { M01, M11, M12 }, { M11, M12, M22 } };
    float sv[3] = { r0, r1, r2 };
    solve3(A, sv);
    if (np <= 4) { sv[0] = 0.f; sv[1] = 0.f; sv[2] = 0.f; }
    for (int a = 0; a < 3; ++a) if (sv[a] != sv[a]) sv[a] = 0.f;
    out[0] = make_float4(c.x, c.y, c.z, sv[0]);
    out[1] = make_float4(t1[0], t1[1], t1[2], sv[1]);
    out[2] = make_float4(t2[0], t2[1], t2[2], sv[2]);
    out[3] = make_float4(n[0], n[1], n[2], (float)np);
}

// sector table [nFeat x 20] (sector of every halfedge of a feature vertex, -1 unused) and the
// sector surfaces FS [4 per sector], one thread per feature vertex
__global__ void k_sector_fit(int nFeat, int nFree, const int* __restrict__ rowptr, const int4* __restrict__ he,
                             const uint8_t* __restrict__ isB1, const float4* __restrict__ pos, const float* __restrict__ fn,
                             const int* __restrict__ srow, int* __restrict__ stab, float4* __restrict__ FS,
                             int* __restrict__ err) {
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nFeat; idx += gridDim.x * blockDim.x) {
        const int vid = nFree + idx, b = rowptr[vid], e = rowptr[vid + 1];
        int* T = stab + (size_t)SECT_TABLE * idx;
        for (int i = 0; i < SECT_TABLE; ++i) T[i] = -1;
        if (e - b > SECT_TABLE) continue;
        T[0] = 0;
        int L[SECT_LIST + 1];
        int sid = 0, nn = 0, lastHE = b, vindex = 1;
        bool last = true;
        for (int i = b + 1; i < e; ++i) {
            const int vdst = he[i].x;
            if (last) { nn = 0; L[nn++] = vid; L[nn++] = he[lastHE].x; }
            if (vdst >= nFree) {
                T[vindex] = sid;
                L[nn++] = vdst;
                sector_fit(L, nn, rowptr, he, pos, fn, FS + 4L * (srow[idx] + sid));
                ++sid;
                nn = 0;
                last = true;
            } else {
                if (nn >= SECT_LIST) { atomicExch(err, 1); break; }
                T[vindex] = sid;
                L[nn++] = vdst;
                last = false;
            }
            ++lastHE;
            ++vindex;
        }
        if (!isB1[vid]) {
            if (last) { nn = 0; L[nn++] = vid; L[nn++] = he[lastHE].x; }
            L[nn++] = he[b].x;
            sector_fit(L, nn, rowptr, he, pos, fn, FS + 4L * (srow[idx] + sid));
        }
    }
}

// 2D mean ratio of (p, a, b) (meanRatioMetricTri2D, dmo/DMOQualityTri.h:243-257)
__device__ __forceinline__ float q2d(float px, float py, float4 a, float4 b) {
    const float e0x = a.x - px, e0y = a.y - py, e1x = b.x - a.x, e1y = b.y - a.y, e2x = px - b.x, e2y = py - b.y;
    const float l = ((e0x * e0x + e0y * e0y) + (e1x * e1x + e1y * e1y)) + (e2x * e2x + e2y * e2y);
    const float area = e0x * e1y - e0y * e1x;
    if (area < 0.f) return area;
    return ((2.f * sqrtf(3.f)) * area) / l;
}

// MODE 0: flat (2D mean ratio; Q 1 / 2: minAngleMetricTri2D / maxAngleMetricTri2D), 1: surface
// triangles, 2: surface quads
template <int MODE, bool SIGNED, int Q>
__device__ __forceinline__ float ring_q1d(const float4* ring, int ne, float px, float py, float pz, float3 n) {
    if (MODE == 0) {
        float q = FLT_MAX;
        for (int i = 0; i < ne; ++i) {
            const float4 a = ring[i], b = ring[i + 1];
            q = fminf(q, Q == 0 ? q2d(px, py, a, b)
                                : (Q == 1 ? tri2d_angle<false>(px, py, a.x, a.y, b.x, b.y)
                                          : tri2d_angle<true>(px, py, a.x, a.y, b.x, b.y)));
        }
        return q;
    }
    return ring_key<MODE == 1 ? 3 : 4, SIGNED, Q>(ring, ne, px, py, pz, n);
}

// localSurfaceEstimation1d (dmo/Surface1D.h:52-93)
__device__ __forceinline__ float3 est1d(const float4* __restrict__ LS1, const float4* __restrict__ X0,
                                        const int* __restrict__ nn, int nnv, const int* surf, int ns, float u) {
    const float4 l0 = LS1[3L * nnv], l1 = LS1[3L * nnv + 1], l2 = LS1[3L * nnv + 2];
    const float w = (l0.w * u) * u;
    const float pwx = (l0.x + u * l1.x) + w * l2.x;
    const float pwy = (l0.y + u * l1.y) + w * l2.y;
    const float pwz = (l0.z + u * l1.z) + w * l2.z;
    const float4 x0 = X0[nnv];
    const float dx = x0.x - pwx, dy = x0.y - pwy, dz = x0.z - pwz;
    const float id = 1.0f / (dot3(dx, dy, dz, dx, dy, dz) + SURF_EPS);
    float isum = id;
    float ax = pwx * id, ay = pwy * id, az = pwz * id;
    for (int i = 0; i < ns; ++i) {
        const int nnN = nn[surf[i]];
        const float4 xn = X0[nnN];
        const float ex = xn.x - pwx, ey = xn.y - pwy, ez = xn.z - pwz;
        const float idn = 1.0f / (dot3(ex, ey, ez, ex, ey, ez) + SURF_EPS);
        isum = isum + idn;
        const float4 m0 = LS1[3L * nnN], m1 = LS1[3L * nnN + 1], m2 = LS1[3L * nnN + 2];
        const float qx = pwx - m0.x, qy = pwy - m0.y, qz = pwz - m0.z;
        const float lu = dot3(qx, qy, qz, m1.x, m1.y, m1.z);
        const float lw = (m0.w * lu) * lu;
        ax = ax + ((m0.x + lu * m1.x) + lw * m2.x) * idn;
        ay = ay + ((m0.y + lu * m1.y) + lw * m2.y) * idn;
        az = az + ((m0.z + lu * m1.z) + lw * m2.z) * idn;
    }
    const float inv = 1.0f / isum;
    return make_float3(ax * inv, ay * inv, az * inv);
}

// The 1D pass over one colour class of feature vertices (k_optimizeHierarchical1DFlat,
// dmo/DMOTriFlatImplCub.h:159-330; k_optimizeHierarchical1D, dmo/DMOTriImplCub.h:205-380,
// dmo/DMOQuadImplCub.h:219-400): lanes 0-7 take the 8 candidates along u of the vertex's curve,
// the first maximum in lane order wins, moves on strict improvement, written when the last
// level's best beats the current position (surfaces: its unsigned ring quality). gate: the
// flat pass runs only while the last minimum quality (stats[*iter]) is positive.
template <int MODE, int Q>
__global__ void __launch_bounds__(SURF_WARPS * 32)
k_dmo_1d(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he,
         const uint8_t* __restrict__ isB1, const float4* __restrict__ X0, const float4* __restrict__ LS1,
         const int* __restrict__ nn, const float* __restrict__ vn, const int* __restrict__ fdeg,
         const uint8_t* __restrict__ opt, int nFree, int v0, int v1, float grid_scale, int maxk,
         const IterStats* __restrict__ stats, const int* __restrict__ iter, const int* __restrict__ list) {
    extern __shared__ float4 s1d[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = v0 + blockIdx.x * SURF_WARPS + warp;
    if (i >= v1) return;
    const int v = list ? list[i] : i;
    if (!opt[v]) return;
    if (stats && !(stats[*iter].min_q > 0.f)) return;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    float4* ring = s1d + (size_t)warp * (2 * maxk + 1 + (maxk + 3) / 4);
    int* surf = reinterpret_cast<int*>(ring + 2 * maxk + 1);
    const float4 c0 = pos[v];
    float md = -FLT_MAX;
    int ns = 0;
    for (int base = 0; base < k; base += 32) {
        const int i = base + lane;
        bool flag = false;
        if (i < k) {
            const int4 h = he[b + i];
            const float4 t = pos[h.x];
            float dx = fabsf(c0.x - t.x), dy = fabsf(c0.y - t.y), dz = fabsf(c0.z - t.z);
            md = fmaxf(md, sqrtf((dx * dx + dy * dy) + dz * dz));
            if (MODE == 2) {
                const float4 t2 = pos[he[h.w].x];
                ring[2 * i] = t;
                ring[2 * i + 1] = t2;
                dx = fabsf(c0.x - t2.x); dy = fabsf(c0.y - t2.y); dz = fabsf(c0.z - t2.z);
                md = fmaxf(md, sqrtf((dx * dx + dy * dy) + dz * dz));
            } else {
                ring[i] = t;
            }
            flag = h.x >= nFree && fdeg[h.x] == 2;
        }
        const unsigned bal = __ballot_sync(FULL, flag);
        if (flag) surf[ns + __popc(bal & ((1u << lane) - 1u))] = he[b + i].x;
        ns += __popc(bal);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) md = fmaxf(md, __shfl_xor_sync(FULL, md, o));
    const bool closed = !isB1[v];
    const int ne = closed ? k : k - 1;
    __syncwarp();
    if (lane == 0 && closed) ring[MODE == 2 ? 2 * k : k] = ring[0];
    __syncwarp();
    const int nnv = nn[v];
    const float4 l0 = LS1[3L * nnv], l1 = LS1[3L * nnv + 1];
    float cu;
    {
        const float qx = c0.x - l0.x, qy = c0.y - l0.y, qz = c0.z - l0.z;
        cu = dot3(qx, qy, qz, l1.x, l1.y, l1.z);
    }
    float3 n = make_float3(0.f, 0.f, 0.f);
    if (MODE != 0) n = make_float3(vn[3L * nnv], vn[3L * nnv + 1], vn[3L * nnv + 2]);
    float cx = c0.x, cy = c0.y, cz = c0.z;
    const float aff = 1.f / 7.f;
    float ds = grid_scale, lastMax = -FLT_MAX;
    for (int d = 0; d < 3; ++d) {
        const float uMax = ds * md, uMin = -ds * md;
        const int i = lane & 7;
        const float u = cu + aff * ((float)i * uMin + (float)(7 - i) * uMax);
        float3 p = make_float3(0.f, 0.f, 0.f);
        float q = -FLT_MAX;
        if (lane < 8) {
            p = est1d(LS1, X0, nn, nnv, surf, ns, u);
            q = ring_q1d<MODE, true, Q>(ring, ne, p.x, p.y, p.z, n);
        }
        float bv = __shfl_sync(FULL, q, 0);
        int bt = 0;
        for (int t = 1; t < 8; ++t) {
            const float qt = __shfl_sync(FULL, q, t);
            if (qt > bv) { bv = qt; bt = t; }
        }
        const float qLast = ring_q1d<MODE, true, Q>(ring, ne, cx, cy, cz, n);
        const float bu = __shfl_sync(FULL, u, bt);
        const float bx = __shfl_sync(FULL, p.x, bt), by = __shfl_sync(FULL, p.y, bt), bz = __shfl_sync(FULL, p.z, bt);
        if (qLast < bv) { cx = bx; cy = by; cz = bz; cu = bu; }
        lastMax = bv;
        ds = ds * (2.f / 7.f);
    }
    const float qOld = ring_q1d<MODE, false, Q>(ring, ne, c0.x, c0.y, c0.z, n);
    if (lane == 0 && qOld < lastMax) pos[v] = make_float4(cx, cy, cz, c0.w);
}

// Boundary-surface pass of a volume mesh (k_optimizeHierarchical2DTet,
// dmo/DMOTetImplCub.h:142-325; k_optimizeHierarchical2DHex, dmo/DMOHexImplCub.h:142-317): the
// surface search of k_dmo_surf over the boundary vertex's surface ring, judged by the key of the
// vertex's volume ring; only while the last minimum quality is positive (dmo/DMOTet.cu:139,
// dmo/DMOHex.cu:152).
template <class R>
__global__ void __launch_bounds__(SURF_WARPS * 32)
k_dmo_surf_vol(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he,
               const int* __restrict__ hf_rowptr, const int4* __restrict__ hf, const float4* __restrict__ X0,
               const float4* __restrict__ LS, const int* __restrict__ nn, int v0, int v1, float grid_scale, int depth,
               int maxkt, int maxks, const int* __restrict__ srow, const int* __restrict__ stab,
               const float4* __restrict__ FS, const float4* __restrict__ Xs, int nFree,
               const IterStats* __restrict__ stats, const int* __restrict__ iter) {
    extern __shared__ float4 sst[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int v = v0 + blockIdx.x * SURF_WARPS + warp;
    if (v >= v1) return;
    if (!(stats[*iter].min_q > 0.f)) return;
    const int b = rowptr[v], ks = rowptr[v + 1] - b;
    if (ks <= 0 || ks > maxks || hf_rowptr[v + 1] - hf_rowptr[v] > maxkt) return;
    float4* co = sst + (size_t)warp * (R::F4 * maxkt + 5 * maxks);
    float4* nbL = co + R::F4 * maxkt;
    float4* nbX = nbL + 4 * maxks;
    const float4 c0 = pos[v];
    R ring;
    if (!ring.stage(pos, hf_rowptr, hf, v, c0, lane, co)) return;
    const float md = ring.md;
    for (int i = lane; i < ks; i += 32) {
        const int nnN = nn[he[b + i].x];
        const float4* Ls = neighbour_surface(v, nnN, LS, rowptr, he, srow, stab, FS, Xs, nFree);
        nbL[4 * i] = Ls[0]; nbL[4 * i + 1] = Ls[1]; nbL[4 * i + 2] = Ls[2]; nbL[4 * i + 3] = Ls[3];
        nbX[i] = X0[nnN];
    }
    __syncwarp();
    const int nnv = nn[v];
    Surf L;
    L.l0 = LS[4L * nnv]; L.l1 = LS[4L * nnv + 1]; L.l2 = LS[4L * nnv + 2]; L.l3 = LS[4L * nnv + 3];
    const float4 x0 = X0[nnv];
    float cu, cv;
    {
        const float dx = c0.x - L.l0.x, dy = c0.y - L.l0.y, dz = c0.z - L.l0.z;
        cu = dot3(dx, dy, dz, L.l1.x, L.l1.y, L.l1.z);
        cv = dot3(dx, dy, dz, L.l2.x, L.l2.y, L.l2.z);
    }
    const float qOld = ring.key(c0.x, c0.y, c0.z);
    const int i1 = lane >> 3, j1 = lane & 7, i2 = i1 + 4;
    const float o1 = (float)(7 - 2 * i1) / 7.f, oj = (float)(7 - 2 * j1) / 7.f, o2 = (float)(7 - 2 * i2) / 7.f;
    float cx = c0.x, cy = c0.y, cz = c0.z;
    float ds = grid_scale, lastMax = -FLT_MAX;
    for (int d = 0; d < depth; ++d) {
        const float S = ds * md;
        const float u1 = fmaf(o1, S, cu), vv = fmaf(oj, S, cv), u2 = fmaf(o2, S, cu);
        const float3 p1 = estimate(L, x0, nbL, nbX, ks, u1, vv);
        const float3 p2 = estimate(L, x0, nbL, nbX, ks, u2, vv);
        const float q1 = ring.key(p1.x, p1.y, p1.z);
        const float q2 = ring.key(p2.x, p2.y, p2.z);
        const bool second = q2 > q1;
        const float val = second ? q2 : q1;
        float bv = __shfl_sync(FULL, val, 0);
        int bt = 0;
        for (int t = 1; t < 32; ++t) {
            const float vt = __shfl_sync(FULL, val, t);
            if (vt > bv) { bv = vt; bt = t; }
        }
        const float qLast = ring.key(cx, cy, cz);
        const float bu = __shfl_sync(FULL, second ? u2 : u1, bt);
        const float bw = __shfl_sync(FULL, vv, bt);
        const float bx = __shfl_sync(FULL, second ? p2.x : p1.x, bt);
        const float by = __shfl_sync(FULL, second ? p2.y : p1.y, bt);
        const float bz = __shfl_sync(FULL, second ? p2.z : p1.z, bt);
        if (qLast < bv) { cx = bx; cy = by; cz = bz; cu = bu; cv = bw; }
        lastMax = bv;
        ds = ds * (2.0f / 7.0f);
    }
    if (lane == 0 && qOld < lastMax) pos[v] = make_float4(cx, cy, cz, c0.w);
}

// 1D pass of the feature vertices on a volume mesh's boundary (k_optimizeHierarchical1DTet,
// dmo/DMOTetImplCub.h:327-494; k_optimizeHierarchical1DHex, dmo/DMOHexImplCub.h:319-487):
// k_dmo_1d with the key of the vertex's volume ring
template <class R>
__global__ void __launch_bounds__(SURF_WARPS * 32)
k_dmo_1d_vol(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he,
             const int* __restrict__ hf_rowptr, const int4* __restrict__ hf, const float4* __restrict__ X0,
             const float4* __restrict__ LS1, const int* __restrict__ nn, const int* __restrict__ fdeg,
             const uint8_t* __restrict__ opt, int nFree, int v0, int v1, float grid_scale, int maxkt, int maxks,
             const IterStats* __restrict__ stats, const int* __restrict__ iter, const int* __restrict__ list) {
    extern __shared__ float4 s1t[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = v0 + blockIdx.x * SURF_WARPS + warp;
    if (i >= v1) return;
    const int v = list ? list[i] : i;
    if (!opt[v]) return;
    if (!(stats[*iter].min_q > 0.f)) return;
    const int b = rowptr[v], ks = rowptr[v + 1] - b;
    if (ks <= 0 || ks > maxks || hf_rowptr[v + 1] - hf_rowptr[v] > maxkt) return;
    float4* co = s1t + (size_t)warp * (R::F4 * maxkt + (maxks + 3) / 4);
    int* surf = reinterpret_cast<int*>(co + R::F4 * maxkt);
    const float4 c0 = pos[v];
    R ring;
    if (!ring.stage(pos, hf_rowptr, hf, v, c0, lane, co)) return;
    const float md = ring.md;
    int ns = 0;
    for (int base = 0; base < ks; base += 32) {
        const int i = base + lane;
        bool flag = false;
        int t = 0;
        if (i < ks) { t = he[b + i].x; flag = t >= nFree && fdeg[t] == 2; }
        const unsigned bal = __ballot_sync(FULL, flag);
        if (flag) surf[ns + __popc(bal & ((1u << lane) - 1u))] = t;
        ns += __popc(bal);
    }
    __syncwarp();
    const int nnv = nn[v];
    const float4 l0 = LS1[3L * nnv], l1 = LS1[3L * nnv + 1];
    float cu;
    {
        const float qx = c0.x - l0.x, qy = c0.y - l0.y, qz = c0.z - l0.z;
        cu = dot3(qx, qy, qz, l1.x, l1.y, l1.z);
    }
    float cx = c0.x, cy = c0.y, cz = c0.z;
    const float aff = 1.f / 7.f;
    float ds = grid_scale, lastMax = -FLT_MAX;
    for (int d = 0; d < 3; ++d) {
        const float uMax = ds * md, uMin = -ds * md;
        const int i = lane & 7;
        const float u = cu + aff * ((float)i * uMin + (float)(7 - i) * uMax);
        float3 p = make_float3(0.f, 0.f, 0.f);
        float q = -FLT_MAX;
        if (lane < 8) {
            p = est1d(LS1, X0, nn, nnv, surf, ns, u);
            q = ring.key(p.x, p.y, p.z);
        }
        float bv = __shfl_sync(FULL, q, 0);
        int bt = 0;
        for (int t = 1; t < 8; ++t) {
            const float qt = __shfl_sync(FULL, q, t);
            if (qt > bv) { bv = qt; bt = t; }
        }
        const float qLast = ring.key(cx, cy, cz);
        const float bu = __shfl_sync(FULL, u, bt);
        const float bx = __shfl_sync(FULL, p.x, bt), by = __shfl_sync(FULL, p.y, bt), bz = __shfl_sync(FULL, p.z, bt);
        if (qLast < bv) { cx = bx; cy = by; cz = bz; cu = bu; }
        lastMax = bv;
        ds = ds * (2.f / 7.f);
    }
    const float qOld = ring.key(c0.x, c0.y, c0.z);
    if (lane == 0 && qOld < lastMax) pos[v] = make_float4(cx, cy, cz, c0.w);
}


}  // namespace

// Sample grids of the GUI's surface views (DMOTriClass::getLocalSurfacePoints /
// getEstimateLocalSurfacePoints, dmo/DMOTri.cu:169-183; kernels dmo/DMOCommon.cu:73-150 and
// dmo/DMOCommon.h:196-276): nu x nv points around the vertex's current local coordinates in
// the frame of its nearest initial vertex's surface, sample idx = i nu + j with u from i and v
// from j, half-extent grid_scale x the ring's largest distance (twice that for the own
// surface). estimate = 0: the own quadric (localToWorldCoords); 1: the blended projection over
// the ring's surfaces, as the search evaluates candidates.
__global__ void k_surface_samples(int estimate_mode, int vid, int nu, int nv, float grid_scale,
                                  const float4* __restrict__ pos, const int* __restrict__ rowptr,
                                  const int4* __restrict__ he, const float4* __restrict__ X0,
                                  const float4* __restrict__ LS, const int* __restrict__ nn, float* __restrict__ out) {
    extern __shared__ float4 ss[];
    __shared__ float s_md;
    const int b = rowptr[vid], k = rowptr[vid + 1] - b;
    float4* nbL = ss;
    float4* nbX = ss + 4 * k;
    const float4 c0 = pos[vid];
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const int nnN = nn[he[b + i].x];
        nbL[4 * i] = LS[4L * nnN]; nbL[4 * i + 1] = LS[4L * nnN + 1];
        nbL[4 * i + 2] = LS[4L * nnN + 2]; nbL[4 * i + 3] = LS[4L * nnN + 3];
        nbX[i] = X0[nnN];
    }
    if (threadIdx.x == 0) {
        float md = -FLT_MAX;
        for (int i = 0; i < k; ++i) {
            const float4 t = pos[he[b + i].x];
            const float dx = t.x - c0.x, dy = t.y - c0.y, dz = t.z - c0.z;
            md = fmaxf(md, sqrtf(dot3(dx, dy, dz, dx, dy, dz)));
        }
        s_md = md;
    }
    __syncthreads();
    const int nnv = nn[vid];
    Surf L;
    L.l0 = LS[4L * nnv]; L.l1 = LS[4L * nnv + 1]; L.l2 = LS[4L * nnv + 2]; L.l3 = LS[4L * nnv + 3];
    const float4 x0 = X0[nnv];
    const float dx = c0.x - L.l0.x, dy = c0.y - L.l0.y, dz = c0.z - L.l0.z;
    const float cu = dot3(dx, dy, dz, L.l1.x, L.l1.y, L.l1.z);
    const float cv = dot3(dx, dy, dz, L.l2.x, L.l2.y, L.l2.z);
    float uMax = grid_scale * s_md, uMin = -grid_scale * s_md;
    float vMax = grid_scale * s_md, vMin = -grid_scale * s_md;
    if (!estimate_mode) { uMin *= 2.f; uMax *= 2.f; vMin *= 2.f; vMax *= 2.f; }
    const float afU = 1.f / (float)(nu - 1), afV = 1.f / (float)(nv - 1);
    for (int idx = threadIdx.x; idx < nu * nv; idx += blockDim.x) {
        const int j = idx % nu, i = idx / nu;
        const float u = cu + afU * ((float)i * uMin + (float)(nu - 1 - i) * uMax);
        const float v = cv + afV * ((float)j * vMin + (float)(nv - 1 - j) * vMax);
        float3 p;
        if (estimate_mode) {
            p = estimate(L, x0, nbL, nbX, k, u, v);
        } else {
            const float w = poly(L.l0, L.l1, L.l2, u, v);
            p = make_float3(((L.l0.x + u * L.l1.x) + v * L.l2.x) + w * L.l3.x,
                            ((L.l0.y + u * L.l1.y) + v * L.l2.y) + w * L.l3.y,
                            ((L.l0.z + u * L.l1.z) + v * L.l2.z) + w * L.l3.z);
        }
        out[3L * idx] = p.x; out[3L * idx + 1] = p.y; out[3L * idx + 2] = p.z;
    }
}

int dmo_surf_max_ring() { return SURF_MAX_RING; }

void launch_surface_samples(const Mesh& m, int estimate_mode, int vid, int nu, int nv, float grid_scale,
                            const float4* X0, const float4* LS, const int* nn, float* out, cudaStream_t s) {
    const size_t smem = (size_t)5 * std::max(m.maxHE, 1) * sizeof(float4);
    k_surface_samples<<<1, 256, smem, s>>>(estimate_mode, vid, nu, nv, grid_scale, m.pos.p, m.he_rowptr.p, m.he.p, X0,
                                           LS, nn, out);
    VSDMO_CHECK_LAUNCH();
}

void launch_surface_fit(const Mesh& m, const float4* pos, float4* LS, int ring, cudaStream_t s) {
    if (m.nSurf <= 0) return;
    k_surface_fit<<<grid_for(m.nSurf, 128), 128, 0, s>>>(m.nSurf, m.he_rowptr.p, m.he.p, pos, m.vn.p, LS, ring == 2 ? 1 : 0);
    VSDMO_CHECK_LAUNCH();
}

void launch_update_nn(const Mesh& m, const float4* X0, int* nn, cudaStream_t s) {
    if (m.nSurf <= 0) return;
    k_update_nn<<<grid_for(m.nSurf, 256), 256, 0, s>>>(m.nSurf, m.nSurf - m.nFeature, m.he_rowptr.p, m.he.p, m.pos.p,
                                                      X0, nn);
    VSDMO_CHECK_LAUNCH();
}

void launch_dmo_surf(const Mesh& m, const DmoLaunch& L, const float4* X0, const float4* LS, const int* nn,
                     const SectorSurfaces* sec, int crit, cudaStream_t s) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    const int maxk = m.maxHE;
    const size_t smem = (size_t)SURF_WARPS * surf_warp_f4(maxk) * sizeof(float4);
    const int blocks = (n + SURF_WARPS - 1) / SURF_WARPS;
    auto k = m.fk == 4 ? (crit == 3 ? k_dmo_surf<4, 3> : k_dmo_surf<4, 0>)
                       : (crit == 1 ? k_dmo_surf<3, 1> : (crit == 2 ? k_dmo_surf<3, 2> : k_dmo_surf<3, 0>));
    k<<<blocks, SURF_WARPS * 32, smem, s>>>(m.pos.p, m.he_rowptr.p, m.he.p, X0, LS, nn, m.vn.p, L.v0, L.v1, L.grid_scale,
                                            L.depth, maxk, sec ? sec->srow : nullptr, sec ? sec->stab : nullptr,
                                            sec ? sec->FS : nullptr, sec ? sec->Xs : nullptr, m.nSurf - m.nFeature);
    VSDMO_CHECK_LAUNCH();
}

void init_feature_state(const Mesh& m, int flat, float4* LS1, int* fdeg, uint8_t* opt, cudaStream_t s) {
    const int nFree = m.nSurf - m.nFeature;
    k_feature_flags<<<grid_for(m.nSurf, 256), 256, 0, s>>>(m.nSurf, nFree, m.he_rowptr.p, m.he.p, m.pos.p, fdeg, opt);
    VSDMO_CHECK_LAUNCH();
    VSDMO_CUDA(cudaMemsetAsync(LS1, 0, sizeof(float4) * 3 * (size_t)m.nSurf, s));
    if (m.nFeature > 0) {
        k_surface_fit_1d<<<grid_for(m.nFeature, 128), 128, 0, s>>>(m.nSurf, nFree, flat, m.he_rowptr.p, m.he.p, m.pos.p,
                                                                   m.vn.p, LS1);
        VSDMO_CHECK_LAUNCH();
    }
}

int build_sectors(const Mesh& m, DBuf<int>& srow, DBuf<int>& stab, DBuf<float4>& FS, cudaStream_t s) {
    const int nFeat = m.nFeature, nFree = m.nSurf - m.nFeature;
    if (nFeat <= 0) return 0;
    DBuf<int> cnt(nFeat, s), err(1, s);
    err.zero();
    srow.alloc(nFeat + 1, s);
    k_sector_count<<<grid_for(nFeat, 128), 128, 0, s>>>(nFeat, nFree, m.he_rowptr.p, m.he.p, m.isB1.p, cnt.p, err.p);
    VSDMO_CHECK_LAUNCH();
    exclusive_scan(cnt.p, srow.p, nFeat, srow.p + nFeat, s);
    const int nSect = read_scalar(srow.p + nFeat, s);
    stab.alloc((size_t)SECT_TABLE * nFeat, s);
    FS.alloc(4 * (size_t)std::max(nSect, 1), s);
    k_sector_fit<<<grid_for(nFeat, 64), 64, 0, s>>>(nFeat, nFree, m.he_rowptr.p, m.he.p, m.isB1.p, m.pos.p, m.fn.p,
                                                   srow.p, stab.p, FS.p, err.p);
    VSDMO_CHECK_LAUNCH();
    if (read_scalar(err.p, s))
        throw Error(VSDMO_E_VALENCE, "a feature vertex has more than 20 halfedges or a sector more than 40 points");
    return nSect;
}

template <class R>
static void surf_vol_launch(const Mesh& m, const DmoLaunch& L, const float4* X0, const float4* LS, const int* nn,
                            const SectorSurfaces* sec, const IterStats* gate_stats, const int* gate_iter,
                            cudaStream_t s) {
    const int n = L.v1 - L.v0;
    const int maxkt = std::max(m.maxTets, 1), maxks = std::max(m.maxHE, 1);
    const size_t smem = (size_t)SURF_WARPS * (R::F4 * maxkt + 5 * maxks) * sizeof(float4);
    k_dmo_surf_vol<R><<<(n + SURF_WARPS - 1) / SURF_WARPS, SURF_WARPS * 32, smem, s>>>(
        m.pos.p, m.he_rowptr.p, m.he.p, m.hf_rowptr.p, m.type == VSDMO_HEX ? m.hh.p : m.hf.p, X0, LS, nn, L.v0, L.v1,
        L.grid_scale, L.depth, maxkt, maxks, sec ? sec->srow : nullptr, sec ? sec->stab : nullptr,
        sec ? sec->FS : nullptr, sec ? sec->Xs : nullptr, m.nSurf - m.nFeature, gate_stats, gate_iter);
    VSDMO_CHECK_LAUNCH();
}

template <class R>
static void vol_1d_launch(const Mesh& m, const DmoLaunch& L, const float4* X0, const float4* LS1, const int* nn,
                          const int* fdeg, const uint8_t* opt, const IterStats* gate_stats, const int* gate_iter,
                          cudaStream_t s, const int* list) {
    const int n = L.v1 - L.v0;
    const int maxkt = std::max(m.maxTets, 1), maxks = std::max(m.maxHE, 1);
    const size_t smem = (size_t)SURF_WARPS * (R::F4 * maxkt + (maxks + 3) / 4) * sizeof(float4);
    k_dmo_1d_vol<R><<<(n + SURF_WARPS - 1) / SURF_WARPS, SURF_WARPS * 32, smem, s>>>(
        m.pos.p, m.he_rowptr.p, m.he.p, m.hf_rowptr.p, m.type == VSDMO_HEX ? m.hh.p : m.hf.p, X0, LS1, nn, fdeg, opt,
        m.nSurf - m.nFeature, L.v0, L.v1, L.grid_scale, maxkt, maxks, gate_stats, gate_iter, list);
    VSDMO_CHECK_LAUNCH();
}

void launch_dmo_surf_vol(const Mesh& m, const DmoLaunch& L, const float4* X0, const float4* LS, const int* nn,
                         const SectorSurfaces* sec, int crit, const IterStats* gate_stats, const int* gate_iter,
                         cudaStream_t s) {
    if (L.v1 <= L.v0) return;
    if (m.type == VSDMO_HEX) surf_vol_launch<HexRing>(m, L, X0, LS, nn, sec, gate_stats, gate_iter, s);
    else if (crit == 1) surf_vol_launch<TetAngleRing<false>>(m, L, X0, LS, nn, sec, gate_stats, gate_iter, s);
    else if (crit == 2) surf_vol_launch<TetAngleRing<true>>(m, L, X0, LS, nn, sec, gate_stats, gate_iter, s);
    else surf_vol_launch<TetRing>(m, L, X0, LS, nn, sec, gate_stats, gate_iter, s);
}

void launch_dmo_1d_vol(const Mesh& m, const DmoLaunch& L, const float4* X0, const float4* LS1, const int* nn,
                       const int* fdeg, const uint8_t* opt, int crit, const IterStats* gate_stats, const int* gate_iter,
                       cudaStream_t s, const int* list) {
    if (L.v1 <= L.v0) return;
    if (m.type == VSDMO_HEX) vol_1d_launch<HexRing>(m, L, X0, LS1, nn, fdeg, opt, gate_stats, gate_iter, s, list);
    else if (crit == 1) vol_1d_launch<TetAngleRing<false>>(m, L, X0, LS1, nn, fdeg, opt, gate_stats, gate_iter, s, list);
    else if (crit == 2) vol_1d_launch<TetAngleRing<true>>(m, L, X0, LS1, nn, fdeg, opt, gate_stats, gate_iter, s, list);
    else vol_1d_launch<TetRing>(m, L, X0, LS1, nn, fdeg, opt, gate_stats, gate_iter, s, list);
}

int surf_vol_max_ring(int elem_type) { return elem_type == VSDMO_HEX ? HEX_SURF_MAX_RING : TET_SURF_MAX_RING; }

void prepare_surf_kernels() {
    const int tet = (int)((size_t)SURF_WARPS * (TetRing::F4 * TET_SURF_MAX_RING + 5 * SURF_MAX_RING) * sizeof(float4));
    const int hex = (int)((size_t)SURF_WARPS * (HexRing::F4 * HEX_SURF_MAX_RING + 5 * SURF_MAX_RING) * sizeof(float4));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_surf_vol<TetRing>, cudaFuncAttributeMaxDynamicSharedMemorySize, tet));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_1d_vol<TetRing>, cudaFuncAttributeMaxDynamicSharedMemorySize, tet));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_surf_vol<HexRing>, cudaFuncAttributeMaxDynamicSharedMemorySize, hex));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_1d_vol<HexRing>, cudaFuncAttributeMaxDynamicSharedMemorySize, hex));
    const int ang = (int)((size_t)SURF_WARPS * (TetAngleRing<false>::F4 * TET_SURF_MAX_RING + 5 * SURF_MAX_RING) *
                          sizeof(float4));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_surf_vol<TetAngleRing<false>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ang));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_surf_vol<TetAngleRing<true>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ang));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_1d_vol<TetAngleRing<false>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ang));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_1d_vol<TetAngleRing<true>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ang));
}

void launch_dmo_1d(const Mesh& m, int mode, const DmoLaunch& L, const float4* X0, const float4* LS1, const int* nn,
                   const int* fdeg, const uint8_t* opt, int crit, const IterStats* gate_stats, const int* gate_iter,
                   cudaStream_t s, const int* list) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    const int maxk = std::max(m.maxHE, 1);
    const size_t smem = (size_t)SURF_WARPS * (2 * maxk + 1 + (maxk + 3) / 4) * sizeof(float4);
    const int blocks = (n + SURF_WARPS - 1) / SURF_WARPS;
    const int nFree = m.nSurf - m.nFeature;
    auto k = mode == 2 ? (crit == 3 ? k_dmo_1d<2, 3> : k_dmo_1d<2, 0>)
           : mode == 1 ? (crit == 1 ? k_dmo_1d<1, 1> : (crit == 2 ? k_dmo_1d<1, 2> : k_dmo_1d<1, 0>))
                       : (crit == 1 ? k_dmo_1d<0, 1> : (crit == 2 ? k_dmo_1d<0, 2> : k_dmo_1d<0, 0>));
    k<<<blocks, SURF_WARPS * 32, smem, s>>>(m.pos.p, m.he_rowptr.p, m.he.p, m.isB1.p, X0, LS1, nn, m.vn.p, fdeg, opt,
                                            nFree, L.v0, L.v1, L.grid_scale, maxk, gate_stats, gate_iter, list);
    VSDMO_CHECK_LAUNCH();
}

}  // namespace vsdmo
