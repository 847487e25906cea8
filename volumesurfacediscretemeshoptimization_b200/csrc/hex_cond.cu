// hex_cond.cu -- DMO of hex interiors under the condition-number quality (hex_cond.cuh), an
// addition to the reference's criteria.
//
// The search is the reference's interior hex search (k_optimizeHierarchicalInnerHex,
// dmo/DMOHexImplCub.h:21-137), as k_dmo_hex runs it for shapeMetricHex: per-axis smallest ring
// distance as the grid extent, 8 x 8 x 8 candidates per level, 128 virtual threads of 4
// candidates whose maxima carry across levels, the lowest thread on ties, strict improvement.
// One block of 128 threads per vertex (the classes of a hex mesh are small: one warp per
// vertex left the SMs with ~4 warps each). The ring is staged in shared memory relative to the vertex and scaled by 2^-e (e from the largest
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
constexpr int HC_THREADS = 128;   // one block per vertex, the reference's block of 128 threads
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

// the ring keys of four candidates (x[0..3], y, z) in one pass over the ring (independent
// chains: the arithmetic of one candidate overlaps the others')
__device__ __forceinline__ void hc_ring_key4(const float4* r, int k, const float* x, float y, float z, float* K) {
#pragma unroll
    for (int a = 0; a < 4; ++a) K[a] = FLT_MAX;
    for (int h = 0; h < k; ++h) {
        float c[7][3];
#pragma unroll
        for (int j = 0; j < 7; ++j) { const float4 t = r[HC_F4 * h + j]; c[j][0] = t.x; c[j][1] = t.y; c[j][2] = t.z; }
        const float ck = r[HC_F4 * h + 7].x;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const float p[3] = { x[a], y, z };
            K[a] = fminf(K[a], hc_halfhex_key(c, ck, p));
        }
    }
}

__device__ __forceinline__ void hc_block_sync() { __syncthreads(); }

// One block of 128 threads per vertex, thread t = the reference's thread t: candidates
// 4t .. 4t+3 (x fastest: x = 4 (t & 1) .. +3, y = (t >> 1) & 7, z = t >> 4).
__global__ void __launch_bounds__(HC_THREADS)
k_dmo_hex_cond(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hh, int v0,
               float grid_scale, int depth, int maxk) {
    extern __shared__ float4 r[];
    __shared__ float red[6][HC_THREADS / 32];
    __shared__ float s_k[HC_THREADS / 32];
    __shared__ int s_i[HC_THREADS / 32];
    __shared__ float s_win[4];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int v = v0 + blockIdx.x;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = pos[v];
    float mx0 = 0.f, mx1 = 0.f, mx2 = 0.f, mn0 = FLT_MAX, mn1 = FLT_MAX, mn2 = FLT_MAX;
    for (int idx = t; idx < 7 * k; idx += HC_THREADS) {
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
    if (lane == 0) { red[0][w] = mx0; red[1][w] = mx1; red[2][w] = mx2; red[3][w] = mn0; red[4][w] = mn1; red[5][w] = mn2; }
    hc_block_sync();
#pragma unroll
    for (int i = 0; i < HC_THREADS / 32; ++i) {
        mx0 = fmaxf(mx0, red[0][i]); mx1 = fmaxf(mx1, red[1][i]); mx2 = fmaxf(mx2, red[2][i]);
        mn0 = fminf(mn0, red[3][i]); mn1 = fminf(mn1, red[4][i]); mn2 = fminf(mn2, red[5][i]);
    }
    const float mm = fmaxf(mx0, fmaxf(mx1, mx2));
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return;   // uniform over the block
    int ex;
    (void)frexpf(mm, &ex);
    const float p2 = exp2_exact(-ex);
    for (int h = t; h < k; h += HC_THREADS) {
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
    hc_block_sync();
    const float sx = scale2(mn0, p2, -ex), sy = scale2(mn1, p2, -ex), sz = scale2(mn2, p2, -ex);
    const int ci = 4 * (t & 1), cj = (t >> 1) & 7, ck = t >> 4;
    float qMax = -FLT_MAX, pX = 0.f, pY = 0.f, pZ = 0.f;
    float dx = 0.f, dy = 0.f, dz = 0.f;
    float ds = grid_scale;
    float qWin = -FLT_MAX;
    for (int level = 0; level < depth; ++level) {
        const float Sx = ds * sx, Sy = ds * sy, Sz = ds * sz;
        const float qLast = hc_ring_key(r, k, dx, dy, dz);
        const float yv = fmaf(hc_offset(cj), Sy, dy), zv = fmaf(hc_offset(ck), Sz, dz);
        float xv[4], K[4];
#pragma unroll
        for (int rr = 0; rr < 4; ++rr) xv[rr] = fmaf(hc_offset(ci + rr), Sx, dx);
        hc_ring_key4(r, k, xv, yv, zv, K);
#pragma unroll
        for (int rr = 0; rr < 4; ++rr)
            if (K[rr] > qMax) { qMax = K[rr]; pX = xv[rr]; pY = yv; pZ = zv; }
        // block arg-max over the carried maxima, the lowest thread on ties
        float bk = qMax;
        int bi = t;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const float ok = __shfl_xor_sync(HC_FULL, bk, o);
            const int oi = __shfl_xor_sync(HC_FULL, bi, o);
            if (ok > bk || (ok == bk && oi < bi)) { bk = ok; bi = oi; }
        }
        if (lane == 0) { s_k[w] = bk; s_i[w] = bi; }
        hc_block_sync();
        bk = s_k[0]; bi = s_i[0];
#pragma unroll
        for (int i = 1; i < HC_THREADS / 32; ++i)
            if (s_k[i] > bk || (s_k[i] == bk && s_i[i] < bi)) { bk = s_k[i]; bi = s_i[i]; }
        if (t == bi) { s_win[0] = pX; s_win[1] = pY; s_win[2] = pZ; }
        hc_block_sync();
        if (qLast < bk) { dx = s_win[0]; dy = s_win[1]; dz = s_win[2]; }
        qWin = bk;
        ds = ds * (2.0f / 7.0f);
        hc_block_sync();   // s_k / s_win are rewritten by the next level
    }
    const float qOld = hc_ring_key(r, k, 0.f, 0.f, 0.f);
    if (t == 0 && qOld < qWin) {
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
    const size_t smem = (size_t)maxk * HC_F4 * sizeof(float4);
    k_dmo_hex_cond<<<n, HC_THREADS, smem, s>>>(m.pos.p, m.hf_rowptr.p, m.hh.p, L.v0, L.grid_scale, L.depth, maxk);
    VSDMO_CHECK_LAUNCH();
}

void prepare_hex_cond_kernels() {}

}  // namespace vsdmo
