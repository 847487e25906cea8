// hex_key.cuh -- the hex ring key of the plain search, shared by the interior search
// (dmo_kernels.cu) and the boundary passes of hex meshes (surf_kernels.cu).
//
// shapeMetricHex (dmo/DMOQualityHex.h:54-71) with the candidate p as corner 0 of a halfhex:
// sub-tets 1, 2, 3 and 6 do not depend on p; sub-tets 0, 4, 5, 7, 8 have a determinant affine
// in p and a Frobenius term quadratic in p. Each halfhex is staged as 43 coefficients (the
// constant part's key and 5 x {g, c, m, C}), relative to the vertex and scaled by 2^-e;
// min_j cbrt(s^2) / A is compared through s^2 / A^3 as a fraction (monotone, no cbrtf).
#pragma once
#include <cuda_runtime.h>

namespace vsdmo {

constexpr int HEX_CO = 44;                      // floats per halfhex (43 used)
constexpr float HEX_EPS = 1.19209e-07f;          // EPSILON of dmo/SurfaceCommon.h

static __device__ __forceinline__ void hcross(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static __device__ __forceinline__ float hdot3(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

static __device__ __forceinline__ void hex_frac(float s, float A, float es, float ea, float& N, float& D, bool& first, bool& zero) {
    if (s < es || A < ea) { zero = true; return; }
    const float num = s * s, den = (A * A) * A;
    if (first) { N = num; D = den; first = false; return; }
    if (num * D < N * den) { N = num; D = den; }
}

// coefficients of one halfhex from its seven corners r (scaled, relative to the vertex)
static __device__ void hex_coeffs(const float r[7][3], float es, float ea, float* out) {
    const float* v1 = r[0]; const float* v2 = r[1]; const float* v3 = r[2]; const float* v4 = r[3];
    const float* v5 = r[4]; const float* v6 = r[5]; const float* v7 = r[6];
    float L0[3], L1[3], L2[3], L3[3], L5[3], L6[3], L7[3], L9[3], L10[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        L0[a] = v5[a] - v4[a]; L1[a] = v6[a] - v5[a]; L2[a] = v7[a] - v6[a]; L3[a] = v7[a] - v4[a];
        L5[a] = v1[a] - v5[a]; L6[a] = v2[a] - v6[a]; L7[a] = v3[a] - v7[a]; L9[a] = v2[a] - v1[a];
        L10[a] = v3[a] - v2[a];
    }
    float N = 0.f, D = 1.f;
    bool first = true, zero = false;
    // constant sub-tets 1 (L1, -L0, L5), 2 (L2, -L1, L6), 3 (-L3, -L2, L7), 6 (-L9, L10, -L6)
    {
        float e[4][3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            e[0][0][a] = L1[a]; e[0][1][a] = -L0[a]; e[0][2][a] = L5[a];
            e[1][0][a] = L2[a]; e[1][1][a] = -L1[a]; e[1][2][a] = L6[a];
            e[2][0][a] = -L3[a]; e[2][1][a] = -L2[a]; e[2][2][a] = L7[a];
            e[3][0][a] = -L9[a]; e[3][1][a] = L10[a]; e[3][2][a] = -L6[a];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float x[3];
            hcross(e[i][1], e[i][2], x);
            const float sd = hdot3(e[i][0], x);
            const float A = (hdot3(e[i][0], e[i][0]) + hdot3(e[i][1], e[i][1])) + hdot3(e[i][2], e[i][2]);
            hex_frac(sd, A, es, ea, N, D, first, zero);
        }
    }
    out[0] = N; out[1] = D; out[2] = zero ? 1.f : 0.f;
    float* co = out + 3;
    float g[3], t1[3], t2[3], t3[3];
    // sub 0: det = (p - v4) . (L0 x L3)
    hcross(L0, L3, g);
    co[0] = g[0]; co[1] = g[1]; co[2] = g[2]; co[3] = -hdot3(v4, g);
    co[4] = -2.f * v4[0]; co[5] = -2.f * v4[1]; co[6] = -2.f * v4[2];
    co[7] = (hdot3(L0, L0) + hdot3(L3, L3)) + hdot3(v4, v4);
    co += 8;
    // sub 4: (v3 - p, v1 - p, v4 - p)
    hcross(v1, v4, t1); hcross(v4, v3, t2); hcross(v3, v1, t3);
    co[0] = -((t1[0] + t2[0]) + t3[0]); co[1] = -((t1[1] + t2[1]) + t3[1]); co[2] = -((t1[2] + t2[2]) + t3[2]);
    co[3] = hdot3(v3, t1);
    co[4] = -2.f * ((v3[0] + v1[0]) + v4[0]); co[5] = -2.f * ((v3[1] + v1[1]) + v4[1]); co[6] = -2.f * ((v3[2] + v1[2]) + v4[2]);
    co[7] = (hdot3(v3, v3) + hdot3(v1, v1)) + hdot3(v4, v4);
    co += 8;
    // sub 5: (p - v1, L9, -L5)
    const float mL5[3] = { -L5[0], -L5[1], -L5[2] };
    hcross(L9, mL5, g);
    co[0] = g[0]; co[1] = g[1]; co[2] = g[2]; co[3] = -hdot3(v1, g);
    co[4] = -2.f * v1[0]; co[5] = -2.f * v1[1]; co[6] = -2.f * v1[2];
    co[7] = hdot3(v1, v1) + (hdot3(L9, L9) + hdot3(L5, L5));
    co += 8;
    // sub 7: (-L10, p - v3, -L7): det = (p - v3) . (L7 x L10)
    hcross(L7, L10, g);
    co[0] = g[0]; co[1] = g[1]; co[2] = g[2]; co[3] = -hdot3(v3, g);
    co[4] = -2.f * v3[0]; co[5] = -2.f * v3[1]; co[6] = -2.f * v3[2];
    co[7] = hdot3(v3, v3) + (hdot3(L10, L10) + hdot3(L7, L7));
    co += 8;
    // sub 8: (Q0 - p, Q1 - p, Q2 + p)
    float Q0[3], Q1[3], Q2[3], a1[3], a2[3], a3[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        Q0[a] = ((v5[a] - v4[a]) + (v6[a] - v7[a])) + (v1[a] + (v2[a] - v3[a]));
        Q1[a] = ((v7[a] - v4[a]) + (v6[a] - v5[a])) + (v3[a] + (v2[a] - v1[a]));
        Q2[a] = ((v1[a] - v5[a]) + (v2[a] - v6[a])) + ((v3[a] - v7[a]) - v4[a]);
    }
    hcross(Q0, Q1, a1); hcross(Q2, Q0, a2); hcross(Q1, Q2, a3);
    co[0] = (a1[0] - a2[0]) - a3[0]; co[1] = (a1[1] - a2[1]) - a3[1]; co[2] = (a1[2] - a2[2]) - a3[2];
    co[3] = hdot3(Q0, a3);
    co[4] = 2.f * ((Q2[0] - Q0[0]) - Q1[0]); co[5] = 2.f * ((Q2[1] - Q0[1]) - Q1[1]); co[6] = 2.f * ((Q2[2] - Q0[2]) - Q1[2]);
    co[7] = (hdot3(Q0, Q0) + hdot3(Q1, Q1)) + hdot3(Q2, Q2);
}

// ring key of one candidate (the current / old position)
static __device__ float hex_key1(const float* co, int k, float x, float y, float z, float es, float ea) {
    const float t1x = x * x, t1y = y * y, t1z = z * z;
    const float t3x = (3.f * x) * x, t3y = (3.f * y) * y, t3z = (3.f * z) * z;
    float N = 0.f, D = 1.f;
    bool first = true, zero = false;
    for (int h = 0; h < k; ++h) {
        const float* c = co + HEX_CO * h;
        if (c[2] != 0.f) zero = true;
        else if (first) { N = c[0]; D = c[1]; first = false; }
        else if (c[0] * D < N * c[1]) { N = c[0]; D = c[1]; }
#pragma unroll
        for (int j = 0; j < 5; ++j) {
            const float* q = c + 3 + 8 * j;
            const bool a3 = (j == 1 || j == 4);
            const float s = fmaf(q[0], x, fmaf(q[1], y, fmaf(q[2], z, q[3])));
            const float A = ((q[7] + fmaf(q[6], z, a3 ? t3z : t1z)) + fmaf(q[5], y, a3 ? t3y : t1y)) +
                            fmaf(q[4], x, a3 ? t3x : t1x);
            hex_frac(s, A, es, ea, N, D, first, zero);
        }
    }
    return zero ? 0.f : N / D;
}

}  // namespace vsdmo
