// hex_cond.cu -- DMO of hex interiors under the condition-number quality (hex_cond.cuh), an
// addition to the reference's criteria.
//
// The search is the reference's interior hex search (k_optimizeHierarchicalInnerHex,
// dmo/DMOHexImplCub.h:21-137), as k_dmo_hex runs it for shapeMetricHex: per-axis smallest ring
// distance as the grid extent, 8 x 8 x 8 candidates per level, 128 virtual threads of 4
// candidates whose maxima carry across levels, the lowest thread on ties, strict improvement.
// One warp per vertex, lane l owns virtual threads 4l .. 4l+3 (fixed z, two y, eight x). The
// ring is staged in shared memory relative to the vertex and scaled by 2^-e (e from the largest
// per-axis ring distance; the key does not change under translation and scaling, and the
// scaling keeps det^2 away from underflow); per halfhex the 7 other corners and the key of its
// four corners that do not touch the vertex.
#include "vsdmo_internal.cuh"
#include "hex_cond.cuh"
#include "tet_key.cuh"
#include <algorithm>
#include <cfloat>

namespace vsdmo {
namespace {

constexpr unsigned HC_FULL = 0xffffffffu;
constexpr int HC_WARPS = 4;
constexpr int HC_MAX_RING = 64;
constexpr int HC_F4 = 8;           // float4 per halfhex: 7 corners, constant key in the 8th

__device__ __forceinline__ float hc_offset(int i) { return (float)(7 - 2 * i) / 7.0f; }

__device__ __forceinline__ float hc_ring_key(const float4* r, int k, float x, float y, float z) {
    const float p[3] = { x, y, z };
    float q = FLT_MAX;
    for (int h = 0; h < k; ++h) {
        float c[7][3];
#pragma unroll
        for (int j = 0; j < 7; ++j) { const float4 t = r[HC_F4 * h + j]; c[j][0] = t.x; c[j][1] = t.y; c[j][2] = t.z; }
        q = fminf(q, hc_halfhex_key(c, r[HC_F4 * h + 7].x, p));
    }
    return q;
}

__global__ void __launch_bounds__(HC_WARPS * 32)
k_dmo_hex_cond(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hh, int v0, int v1,
               float grid_scale, int depth, int maxk) {
    extern __shared__ float4 hc_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int v = v0 + blockIdx.x * HC_WARPS + w;
    if (v >= v1) return;
    float4* r = hc_smem + (size_t)w * maxk * HC_F4;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = pos[v];
    float mx0 = 0.f, mx1 = 0.f, mx2 = 0.f, mn0 = FLT_MAX, mn1 = FLT_MAX, mn2 = FLT_MAX;
    for (int idx = lane; idx < 7 * k; idx += 32) {
        const int h = idx / 7, c = idx % 7;
        const int4 q = hh[2 * (b + h) + (c >> 2)];
        const int cc = c & 3;
        const float4 p = pos[cc == 0 ? q.x : (cc == 1 ? q.y : (cc == 2 ? q.z : q.w))];
        const float d0 = fabsf(p.x - c0.x), d1 = fabsf(p.y - c0.y), d2 = fabsf(p.z - c0.z);
        mx0 = fmaxf(mx0, d0); mx1 = fmaxf(mx1, d1); mx2 = fmaxf(mx2, d2);
        mn0 = fminf(mn0, d0); mn1 = fminf(mn1, d1); mn2 = fminf(mn2, d2);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        mx0 = fmaxf(mx0, __shfl_xor_sync(HC_FULL, mx0, o)); mx1 = fmaxf(mx1, __shfl_xor_sync(HC_FULL, mx1, o));
        mx2 = fmaxf(mx2, __shfl_xor_sync(HC_FULL, mx2, o)); mn0 = fminf(mn0, __shfl_xor_sync(HC_FULL, mn0, o));
        mn1 = fminf(mn1, __shfl_xor_sync(HC_FULL, mn1, o)); mn2 = fminf(mn2, __shfl_xor_sync(HC_FULL, mn2, o));
    }
    const float mm = fmaxf(mx0, fmaxf(mx1, mx2));
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return;
    int ex;
    (void)frexpf(mm, &ex);
    const float p2 = exp2_exact(-ex);
    for (int h = lane; h < k; h += 32) {
        const int4 qa = hh[2 * (b + h)], qb = hh[2 * (b + h) + 1];
        const int us[7] = { qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z };
        float c[7][3];
#pragma unroll
        for (int j = 0; j < 7; ++j) {
            const float4 p = pos[us[j]];
            c[j][0] = scale2(p.x - c0.x, p2, -ex); c[j][1] = scale2(p.y - c0.y, p2, -ex); c[j][2] = scale2(p.z - c0.z, p2, -ex);
            r[HC_F4 * h + j] = make_float4(c[j][0], c[j][1], c[j][2], 0.f);
        }
        r[HC_F4 * h + 7] = make_float4(hc_const_key(c), 0.f, 0.f, 0.f);
    }
    __syncwarp();
    const float sx = scale2(mn0, p2, -ex), sy = scale2(mn1, p2, -ex), sz = scale2(mn2, p2, -ex);
    const int kz = lane >> 2, j0 = 2 * (lane & 3);
    float qMax[4] = { -FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX };
    float pX[4] = { 0.f, 0.f, 0.f, 0.f }, pY[4] = { 0.f, 0.f, 0.f, 0.f }, pZ[4] = { 0.f, 0.f, 0.f, 0.f };
    float dx = 0.f, dy = 0.f, dz = 0.f;
    float ds = grid_scale;
    float qWin = -FLT_MAX;
    for (int level = 0; level < depth; ++level) {
        const float Sx = ds * sx, Sy = ds * sy, Sz = ds * sz;
        const float qLast = hc_ring_key(r, k, dx, dy, dz);
        const float z = fmaf(hc_offset(kz), Sz, dz);
        const float y[2] = { fmaf(hc_offset(j0), Sy, dy), fmaf(hc_offset(j0 + 1), Sy, dy) };
        // virtual thread 4 lane + t takes x 4 (t & 1) .. +3 at y[t >> 1]; its maximum carries
        // across levels (candidates in index order, strict >)
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float yv = y[t >> 1];
#pragma unroll 1
            for (int rr = 0; rr < 4; ++rr) {
                const float xv = fmaf(hc_offset(4 * (t & 1) + rr), Sx, dx);
                const float key = hc_ring_key(r, k, xv, yv, z);
                if (key > qMax[t]) { qMax[t] = key; pX[t] = xv; pY[t] = yv; pZ[t] = z; }
            }
        }
        float bk = qMax[0];
        int bi = 4 * lane;
#pragma unroll
        for (int t = 1; t < 4; ++t)
            if (qMax[t] > bk) { bk = qMax[t]; bi = 4 * lane + t; }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const float ok = __shfl_xor_sync(HC_FULL, bk, o);
            const int oi = __shfl_xor_sync(HC_FULL, bi, o);
            if (ok > bk || (ok == bk && oi < bi)) { bk = ok; bi = oi; }
        }
        const int src = bi >> 2, tt = bi & 3;
        const float wx = __shfl_sync(HC_FULL, tt == 0 ? pX[0] : (tt == 1 ? pX[1] : (tt == 2 ? pX[2] : pX[3])), src);
        const float wy = __shfl_sync(HC_FULL, tt == 0 ? pY[0] : (tt == 1 ? pY[1] : (tt == 2 ? pY[2] : pY[3])), src);
        const float wz = __shfl_sync(HC_FULL, tt == 0 ? pZ[0] : (tt == 1 ? pZ[1] : (tt == 2 ? pZ[2] : pZ[3])), src);
        if (qLast < bk) { dx = wx; dy = wy; dz = wz; }
        qWin = bk;
        ds = ds * (2.0f / 7.0f);
    }
    const float qOld = hc_ring_key(r, k, 0.f, 0.f, 0.f);
    if (lane == 0 && qOld < qWin) {
        const float e2 = exp2_exact(ex);
        pos[v] = make_float4(c0.x + scale2(dx, e2, ex), c0.y + scale2(dy, e2, ex), c0.z + scale2(dz, e2, ex), c0.w);
    }
}

}  // namespace

int dmo_hex_cond_max_ring() { return HC_MAX_RING; }

void launch_dmo_hex_cond(const Mesh& m, const DmoLaunch& L, cudaStream_t s) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    const int maxk = std::max(m.maxTets, 1);
    const size_t smem = (size_t)HC_WARPS * maxk * HC_F4 * sizeof(float4);
    k_dmo_hex_cond<<<(n + HC_WARPS - 1) / HC_WARPS, HC_WARPS * 32, smem, s>>>(m.pos.p, m.hf_rowptr.p, m.hh.p, L.v0, L.v1,
                                                                            L.grid_scale, L.depth, maxk);
    VSDMO_CHECK_LAUNCH();
}

void prepare_hex_cond_kernels() {
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_hex_cond, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    HC_WARPS * HC_MAX_RING * HC_F4 * (int)sizeof(float4)));
}

}  // namespace vsdmo
