// angle.cu -- DMO with the reference's angle criteria (MIN_ANGLE, MAX_ANGLE) for tet interiors
// and flat triangle meshes.
//
// The searches are those of the mean-ratio kernels (k_optimizeHierarchicalInnerTet,
// dmo/DMOTetImplCub.h:21-137; k_optimizeHierarchical2DFlat, dmo/DMOTriFlatImplCub.h:24-152):
// the same candidate grids, tie rules (lowest candidate index; p2 on a 2D tie) and write rules;
// the ring key is the literal element metric of angle_metrics.cuh (acosf per element and
// candidate; no algebraic shortcut exists for angles), minimised over the ring. One warp per
// vertex; the ring is staged in shared memory relative to the vertex.
#include "vsdmo_internal.cuh"
#include "angle_metrics.cuh"
#include <cfloat>

namespace vsdmo {
namespace {

constexpr unsigned AFULL = 0xffffffffu;
constexpr int AW = 4;                 // warps per block
constexpr int ATET_MAX_RING = 256;
constexpr int ATRI_MAX_RING = 256;

__device__ __forceinline__ float aoff(int i) { return (float)(7 - 2 * i) / 7.0f; }

__device__ __forceinline__ void a_argmax(float& k, int& i) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float ok = __shfl_xor_sync(AFULL, k, o);
        const int oi = __shfl_xor_sync(AFULL, i, o);
        if (ok > k || (ok == k && oi < i)) { k = ok; i = oi; }
    }
}
__device__ __forceinline__ float a_wmax(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(AFULL, v, o));
    return v;
}

template <bool MAXA>
__device__ float tet_ring_angle(const float4* ring, int k, float x, float y, float z) {
    const float p[3] = { x, y, z };
    float q = FLT_MAX;
    for (int t = 0; t < k; ++t) {
        const float4 a = ring[3 * t], b = ring[3 * t + 1], c = ring[3 * t + 2];
        const float pa[3] = { a.x, a.y, a.z }, pb[3] = { b.x, b.y, b.z }, pc[3] = { c.x, c.y, c.z };
        q = fminf(q, tet_angle<MAXA>(p, pa, pb, pc));
    }
    return q;
}

template <bool MAXA>
__global__ void __launch_bounds__(AW * 32)
k_dmo_tet_angle(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hf, int v0, int v1,
                float grid_scale, int depth, int maxk) {
    extern __shared__ float4 asm_ring[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int v = v0 + blockIdx.x * AW + w;
    if (v >= v1) return;
    float4* ring = asm_ring + (size_t)w * maxk * 3;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = pos[v];
    float mx = 0.f, my = 0.f, mz = 0.f;
    for (int t = lane; t < k; t += 32) {
        const int4 h = hf[b + t];
        const int ids[3] = { h.x, h.y, h.z };
        for (int j = 0; j < 3; ++j) {
            const float4 q = pos[ids[j]];
            const float4 r = make_float4(q.x - c0.x, q.y - c0.y, q.z - c0.z, 0.f);
            ring[3 * t + j] = r;
            mx = fmaxf(mx, fabsf(r.x)); my = fmaxf(my, fabsf(r.y)); mz = fmaxf(mz, fabsf(r.z));
        }
    }
    mx = a_wmax(mx); my = a_wmax(my); mz = a_wmax(mz);
    __syncwarp();
    float cx = 0.f, cy = 0.f, cz = 0.f;
    float qLast = tet_ring_angle<MAXA>(ring, k, 0.f, 0.f, 0.f);
    bool moved = false;
    float ds = grid_scale;
    for (int level = 0; level < depth; ++level) {
        const float Sx = ds * mx, Sy = ds * my, Sz = ds * mz;
        float bk = -FLT_MAX;
        int bi = 1 << 30;
        for (int idx = lane; idx < 512; idx += 32) {
            const float x = fmaf(aoff(idx & 7), Sx, cx), y = fmaf(aoff((idx >> 3) & 7), Sy, cy), z = fmaf(aoff(idx >> 6), Sz, cz);
            const float q = tet_ring_angle<MAXA>(ring, k, x, y, z);
            if (q > bk || bi == (1 << 30)) { bk = q; bi = idx; }
        }
        a_argmax(bk, bi);
        if (bi < 512 && qLast < bk) {
            cx = fmaf(aoff(bi & 7), Sx, cx); cy = fmaf(aoff((bi >> 3) & 7), Sy, cy); cz = fmaf(aoff(bi >> 6), Sz, cz);
            qLast = bk;
            moved = true;
        }
        ds = ds * (2.0f / 7.0f);
    }
    if (moved && lane == 0) pos[v] = make_float4(c0.x + cx, c0.y + cy, c0.z + cz, c0.w);
}

template <bool MAXA>
__device__ float tri_ring_angle(const float2* ring, int k, float x, float y) {
    float q = FLT_MAX;
    for (int t = 0; t < k; ++t) {
        const float2 a = ring[t], b = ring[t + 1 == k ? 0 : t + 1];
        q = fminf(q, tri2d_angle<MAXA>(x, y, a.x, a.y, b.x, b.y));
    }
    return q;
}

template <bool MAXA>
__global__ void __launch_bounds__(AW * 32)
k_dmo_tri2d_angle(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he, int v0, int v1,
                  float grid_scale, int depth, int maxk) {
    extern __shared__ float2 asm_fan[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int v = v0 + blockIdx.x * AW + w;
    if (v >= v1) return;
    float2* ring = asm_fan + (size_t)w * maxk;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = pos[v];
    float mx = 0.f, my = 0.f;
    for (int t = lane; t < k; t += 32) {
        const float4 q = pos[he[b + t].x];
        const float2 r = make_float2(q.x - c0.x, q.y - c0.y);
        ring[t] = r;
        mx = fmaxf(mx, fabsf(r.x)); my = fmaxf(my, fabsf(r.y));
    }
    mx = a_wmax(mx); my = a_wmax(my);
    __syncwarp();
    // lane t: (i1 = t / 8, j1 = t % 8) and (i1 + 4, j1); a lane's value is the larger key, its
    // point the first candidate's only when that key is strictly larger
    const int i1 = lane >> 3, j1 = lane & 7;
    float cx = 0.f, cy = 0.f;
    const float qOld = tri_ring_angle<MAXA>(ring, k, 0.f, 0.f);
    float qLast = qOld, lastMax = -FLT_MAX;
    float ds = grid_scale;
    for (int level = 0; level < depth; ++level) {
        const float Sx = ds * mx, Sy = ds * my;
        const float x1 = fmaf(aoff(i1), Sx, cx), x2 = fmaf(aoff(i1 + 4), Sx, cx), y = fmaf(aoff(j1), Sy, cy);
        const float q1 = tri_ring_angle<MAXA>(ring, k, x1, y), q2 = tri_ring_angle<MAXA>(ring, k, x2, y);
        float val = q1;
        if (q2 > q1) val = q2;
        const float selx = q1 > q2 ? x1 : x2;
        float bv = val;
        int bl = lane;
        a_argmax(bv, bl);
        if (qLast < bv) {
            cx = __shfl_sync(AFULL, selx, bl);
            cy = __shfl_sync(AFULL, y, bl);
            qLast = bv;
        }
        lastMax = bv;
        ds = ds * (2.0f / 7.0f);
    }
    if (qOld < lastMax && lane == 0) pos[v] = make_float4(c0.x + cx, c0.y + cy, c0.z, c0.w);
}

}  // namespace

int dmo_angle_max_ring(int elem_type) { return elem_type == VSDMO_TET ? ATET_MAX_RING : ATRI_MAX_RING; }

void launch_dmo_angle(const Mesh& m, const DmoLaunch& L, bool max_angle, cudaStream_t s) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    const int blocks = (n + AW - 1) / AW;
    if (m.type == VSDMO_TET) {
        const int maxk = std::max(m.maxTets, 1);
        const size_t smem = (size_t)AW * maxk * 3 * sizeof(float4);
        if (max_angle)
            k_dmo_tet_angle<true><<<blocks, AW * 32, smem, s>>>(m.pos.p, m.hf_rowptr.p, m.hf.p, L.v0, L.v1, L.grid_scale, L.depth, maxk);
        else
            k_dmo_tet_angle<false><<<blocks, AW * 32, smem, s>>>(m.pos.p, m.hf_rowptr.p, m.hf.p, L.v0, L.v1, L.grid_scale, L.depth, maxk);
    } else {
        const int maxk = std::max(m.maxHE, 1);
        const size_t smem = (size_t)AW * maxk * sizeof(float2);
        if (max_angle)
            k_dmo_tri2d_angle<true><<<blocks, AW * 32, smem, s>>>(m.pos.p, m.he_rowptr.p, m.he.p, L.v0, L.v1, L.grid_scale, L.depth, maxk);
        else
            k_dmo_tri2d_angle<false><<<blocks, AW * 32, smem, s>>>(m.pos.p, m.he_rowptr.p, m.he.p, L.v0, L.v1, L.grid_scale, L.depth, maxk);
    }
    VSDMO_CHECK_LAUNCH();
}

void prepare_angle_kernels() {
    const int tet = AW * ATET_MAX_RING * 3 * (int)sizeof(float4);
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_tet_angle<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tet));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_tet_angle<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tet));
}

}  // namespace vsdmo
