// dmo_kernels.cu -- the DMO grid search and the quality reductions.
//
// Grid search (one colour class per launch, one warp per free vertex). Replaces
//   k_optimizeHierarchicalInnerTet<128>  dmo/DMOTetImplCub.h:21-137  (tet interior)
//   k_optimizeHierarchical2DFlat<32>     dmo/DMOTriFlatImplCub.h:24-152 (flat triangles)
// Same search as the reference: N x N (x N) candidates per level centred on the current
// position, half-extent grid_scale * (per-axis max ring distance) shrinking by 2/(N-1) per
// level, the vertex moved to the best candidate (largest ring minimum of the mean ratio,
// lowest linear index x-fastest on ties) when it strictly beats the current position, and
// written back only on improvement. What differs is the arithmetic:
//   * the ring is staged as per-element coefficients in shared memory: relative to the
//     vertex and scaled by an exact power of two, the tet determinant is affine in the
//     candidate p (det = d0 - n.p) and the sum of the six squared edge lengths is
//     quadratic (L = C - 2 s.p + 3|p|^2); the flat-triangle area and edge sum likewise;
//   * each lane owns 16 (tet) or 2 (2D) candidates of a separable grid, so one element
//     costs 3 FMAs + a compare per candidate instead of a full metric evaluation;
//   * the ring minimum is compared through the monotone transform det^2/L^3 (A/L in 2D),
//     kept as a fraction and compared by cross-multiplication (no cbrt or divide per
//     element); inverted elements key the ring by their most negative det / area, the
//     analogue of the reference returning the negative volume / area;
//   * the block-wide cub::ArgMax becomes a warp butterfly on (key, candidate index).
// The library is compiled with --fmad=false: the only fused multiply-adds are the written
// fmaf() calls, so the CPU restatement in oracle/or_dmo.c reproduces every bit.
//
// Quality reductions: k_quality_stats replaces k_updateCurrentQualities + k_findMinimumQuality
// (dmo/DMOTet.cu:45-67) in one deterministic launch; k_quality_histogram and
// k_element_qualities replace k_qualityHistogram / k_getElementQualities (dmo/DMOTet.cu:31-43,69-75).
#include "vsdmo_internal.cuh"
#include "tc_gemm.cuh"
#include "angle_metrics.cuh"
#include "tet_key.cuh"
#include "hex_key.cuh"
#include "hex_cond.cuh"
#include "quad_cond.cuh"
#include <cfloat>
#include <cuda_bf16.h>
#include <algorithm>

namespace vsdmo {
namespace {

constexpr int NQ = 8;
constexpr unsigned FULL = 0xffffffffu;

// packed position of feature (row, col) in the network's 96-column input operand
__device__ __forceinline__ size_t learned_pk_off(long row, int col) { return tc::pk_off(row, col, 96); }
// launch shape of the tet kernel: 4 warps per block, measured fastest on B200 against 2 and 8
#ifndef TET_WARPS_CFG
#define TET_WARPS_CFG 4
#endif
#ifndef TET_MIN_BLOCKS
#define TET_MIN_BLOCKS 0
#endif
#ifndef TET_SPLIT_Y
#define TET_SPLIT_Y 0
#endif
constexpr int TET_WARPS = TET_WARPS_CFG;
constexpr int TRI_WARPS = 4;
constexpr int TET_MAX_RING = 512;
constexpr int TRI_MAX_RING = 256;

// candidate offsets (N-1-2i)/(N-1): i = 0 is +extent, i = N-1 is -extent (DMOTetImplCub.h:101-103)
__device__ __forceinline__ float grid_offset(int i) {
    switch (i) {
    case 0: return 7.0f / 7.0f;
    case 1: return 5.0f / 7.0f;
    case 2: return 3.0f / 7.0f;
    case 3: return 1.0f / 7.0f;
    case 4: return -1.0f / 7.0f;
    case 5: return -3.0f / 7.0f;
    case 6: return -5.0f / 7.0f;
    default: return -7.0f / 7.0f;
    }
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

// (key, index): larger key wins, equal keys -> lower index (cub::ArgMax semantics)
__device__ __forceinline__ void warp_argmax(float& k, int& i) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        float ok = __shfl_xor_sync(FULL, k, o);
        int oi = __shfl_xor_sync(FULL, i, o);
        if (ok > k || (ok == k && oi < i)) { k = ok; i = oi; }
    }
}

// Ring minimum of the lane's candidates (fixed x, NJ y values, all NQ z values) over the k
// tets of the ring; returns the lane's best (key, linear index), strict > in index order.
template <int NJ>
__device__ __forceinline__ void tet_lane_best(const float4* __restrict__ co, int k, float x, const float* y,
                                              const float* z, const float* tz, int ci, int cj, int jbase,
                                              float& bk, int& bi) {
    const float tx = (3.0f * x) * x;
    float ty[NJ];
#pragma unroll
    for (int jj = 0; jj < NJ; ++jj) ty[jj] = (3.0f * y[jj]) * y[jj];
    float N[NJ][NQ], D[NJ][NQ], dm[NJ][NQ];
    {
        const float4 K0 = co[0], K1 = co[1];
        const float detA = fmaf(K0.x, x, K0.w);
        const float LA = K1.w + fmaf(K1.x, x, tx);
#pragma unroll
        for (int jj = 0; jj < NJ; ++jj) {
            const float detB = fmaf(K0.y, y[jj], detA), LB = LA + fmaf(K1.y, y[jj], ty[jj]);
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const float det = fmaf(K0.z, z[q], detB), L = LB + fmaf(K1.z, z[q], tz[q]);
                N[jj][q] = det * det; D[jj][q] = (L * L) * L; dm[jj][q] = det;
            }
        }
    }
    for (int t = 1; t < k; ++t) {
        const float4 K0 = co[2 * t], K1 = co[2 * t + 1];
        const float detA = fmaf(K0.x, x, K0.w);
        const float LA = K1.w + fmaf(K1.x, x, tx);
        float detB[NJ], LB[NJ];
#pragma unroll
        for (int jj = 0; jj < NJ; ++jj) { detB[jj] = fmaf(K0.y, y[jj], detA); LB[jj] = LA + fmaf(K1.y, y[jj], ty[jj]); }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const float lz = fmaf(K1.z, z[q], tz[q]);
#pragma unroll
            for (int jj = 0; jj < NJ; ++jj) {
                const float det = fmaf(K0.z, z[q], detB[jj]), L = LB[jj] + lz;
                const float num = det * det, den = (L * L) * L;
                if (num * D[jj][q] < N[jj][q] * den) { N[jj][q] = num; D[jj][q] = den; }
                dm[jj][q] = fminf(dm[jj][q], det);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
#pragma unroll
        for (int jj = 0; jj < NJ; ++jj) {
            const float key = dm[jj][q] < 0.f ? dm[jj][q] : N[jj][q] / D[jj][q];
            const int idx = ci + 8 * (cj + 4 * (jbase + jj)) + 64 * q;
            if (key > bk || (key == bk && idx < bi)) { bk = key; bi = idx; }
        }
    }
}

// ---- candidate filter of the tet search --------------------------------------------------------
// The ring key of a candidate is a minimum over the ring's tets, so the minimum over any subset
// of them bounds it from above. A level can only move the vertex to a candidate whose key
// beats qLast, so a candidate whose key over a few tets is already below qLast can never be
// chosen: the search evaluates the TET_CRIT tets with the smallest keys at the level's centre
// for all 512 candidates, keeps the candidates that are not below qLast (with a relative
// margin of 2^-14 that covers the rounding of the fraction comparisons), and evaluates the
// full ring only for those, in the same operations and tet order as the plain search. The
// winner, and whether the vertex moves, are the same as without the filter: every candidate
// that beats qLast survives, and no discarded candidate can tie with or exceed one that does.
#ifndef TET_CRIT_CFG
#define TET_CRIT_CFG 6
#endif
constexpr int TET_CRIT = TET_CRIT_CFG;   // tets of the filter
constexpr int TET_LIST = 256;    // survivors per warp evaluated from a list (more: full search)

// (num, den, det) of tet t at (x, y, z): the operations of tet_key1
__device__ __forceinline__ float tet_piece_key(const float4* __restrict__ co, int t, float x, float y, float z) {
    const float4 c0 = co[2 * t], c1 = co[2 * t + 1];
    const float tx = (3.0f * x) * x, ty = (3.0f * y) * y, tz = (3.0f * z) * z;
    const float det = fmaf(c0.z, z, fmaf(c0.y, y, fmaf(c0.x, x, c0.w)));
    const float L = ((c1.w + fmaf(c1.x, x, tx)) + fmaf(c1.y, y, ty)) + fmaf(c1.z, z, tz);
    return det < 0.f ? det : (det * det) / ((L * L) * L);
}

// The TET_CRIT tets of smallest key at (x, y, z), the same on all lanes. Any choice of tets gives
// an exact filter (the key over any subset bounds the ring key from above), so the choice needs
// no exact arithmetic: a ring of up to 32 tets keys each tet once on its lane (fast division),
// orders the keys as unsigned integers whose low 5 bits are the tet index and takes the minimum
// TET_CRIT times with one warp reduction each. Larger rings scan their tets per round.
__device__ __forceinline__ unsigned tet_order_key(float key, int t) {
    const unsigned b = __float_as_uint(key);
    const unsigned o = (b & 0x80000000u) ? ~b : (b | 0x80000000u);   // float order as unsigned order
    return (o & ~31u) | (unsigned)t;
}

__device__ __forceinline__ float tet_piece_key_fast(const float4* __restrict__ co, int t, float x, float y, float z) {
    const float4 c0 = co[2 * t], c1 = co[2 * t + 1];
    const float tx = (3.0f * x) * x, ty = (3.0f * y) * y, tz = (3.0f * z) * z;
    const float det = fmaf(c0.z, z, fmaf(c0.y, y, fmaf(c0.x, x, c0.w)));
    const float L = ((c1.w + fmaf(c1.x, x, tx)) + fmaf(c1.y, y, ty)) + fmaf(c1.z, z, tz);
    return det < 0.f ? det : __fdividef(det * det, (L * L) * L);
}

__device__ __forceinline__ void tet_critical(const float4* __restrict__ co, int k, float x, float y, float z, int lane,
                                             int (&crit)[TET_CRIT]) {
    if (k <= 32) {
        unsigned mine = lane < k ? tet_order_key(tet_piece_key_fast(co, lane, x, y, z), lane) : 0xffffffffu;
#pragma unroll
        for (int r = 0; r < TET_CRIT; ++r) {
            const unsigned m = __reduce_min_sync(FULL, mine);
            const int t = (int)(m & 31u);
            crit[r] = t < k ? t : 0;
            if (lane == t) mine = 0xffffffffu;
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < TET_CRIT; ++r) {
        unsigned best = 0xffffffffu;
        int bt = 0;
        for (int t = lane; t < k; t += 32) {
            bool used = false;
#pragma unroll
            for (int q = 0; q < r; ++q) used |= (crit[q] == t);
            if (used) continue;
            const unsigned kt = tet_order_key(tet_piece_key_fast(co, t, x, y, z), t & 31);
            if (kt < best || (kt == best && t < bt)) { best = kt; bt = t; }
        }
        // the warp's smallest (key, tet) pair: reduce the key, then the tet among the lanes holding it
        const unsigned m = __reduce_min_sync(FULL, best);
        const unsigned tt = __reduce_min_sync(FULL, best == m ? (unsigned)bt : 0xffffffffu);
        crit[r] = tt < (unsigned)k ? (int)tt : 0;
    }
}

// the lane's 16 candidates (fixed x, y[2], z[8]) over the critical tets: bit jj * 8 + q set when
// the candidate survives (its key over the subset is not below thr). Used when thr <= 0 (the
// ring has an inverted tet, whose key is its det); tet_filter_pos covers thr > 0.
#ifndef TET_FILTER_NEG_INLINE
#define TET_FILTER_NEG_INLINE 1
#endif
#if TET_FILTER_NEG_INLINE
__device__ __forceinline__
#else
__device__ __noinline__
#endif
unsigned tet_filter(const float4* __restrict__ co, const int (&crit)[TET_CRIT], int m,
                                               float x, const float* y, const float* z, const float* tz, float thr) {
    const float tx = (3.0f * x) * x;
    const float ty[2] = { (3.0f * y[0]) * y[0], (3.0f * y[1]) * y[1] };
    float N[2][NQ], D[2][NQ], dm[2][NQ];
#pragma unroll
    for (int r = 0; r < TET_CRIT; ++r) {
        if (r >= m) break;
        const int t = crit[r];
        const float4 K0 = co[2 * t], K1 = co[2 * t + 1];
        const float detA = fmaf(K0.x, x, K0.w);
        const float LA = K1.w + fmaf(K1.x, x, tx);
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            const float detB = fmaf(K0.y, y[jj], detA), LB = LA + fmaf(K1.y, y[jj], ty[jj]);
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const float det = fmaf(K0.z, z[q], detB), L = LB + fmaf(K1.z, z[q], tz[q]);
                const float num = det * det, den = (L * L) * L;
                if (r == 0) { N[jj][q] = num; D[jj][q] = den; dm[jj][q] = det; continue; }
                if (num * D[jj][q] < N[jj][q] * den) { N[jj][q] = num; D[jj][q] = den; }
                dm[jj][q] = fminf(dm[jj][q], det);
            }
        }
    }
    unsigned alive = 0;
#pragma unroll
    for (int jj = 0; jj < 2; ++jj)
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            // key < thr, with the fraction compared by cross-multiplication (its rounding is
            // far inside thr's margin)
            const bool below = dm[jj][q] < 0.f ? dm[jj][q] < thr : N[jj][q] < thr * D[jj][q];
            if (!below) alive |= 1u << (jj * 8 + q);
        }
    return alive;
}

// thr > 0: a candidate survives when every critical tet has det > 0 and det^2 >= thr L^3, tested
// as min over the tets of min(det, det^2 - thr L^3) > 0 -- one running minimum instead of a
// fraction and a det. det, det^2 and L^3 are the values the fraction would be formed from, and
// the fma rounds det^2 - thr L^3 once, so a tet whose key det^2 / L^3 is at least the current
// key (thr lies 2^-14 of it lower) gives a positive value: every candidate that can beat the
// current key survives.
__device__ __forceinline__ unsigned tet_filter_pos(const float4* __restrict__ co, const int (&crit)[TET_CRIT], int m,
                                                   float x, const float* y, const float* z, const float* tz,
                                                   float thr) {
    const float tx = (3.0f * x) * x;
    const float ty[2] = { (3.0f * y[0]) * y[0], (3.0f * y[1]) * y[1] };
    float s[2][NQ];
#pragma unroll
    for (int r = 0; r < TET_CRIT; ++r) {
        if (r >= m) break;
        const int t = crit[r];
        const float4 K0 = co[2 * t], K1 = co[2 * t + 1];
        const float detA = fmaf(K0.x, x, K0.w);
        const float LA = K1.w + fmaf(K1.x, x, tx);
        float lz[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) lz[q] = fmaf(K1.z, z[q], tz[q]);
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            const float detB = fmaf(K0.y, y[jj], detA), LB = LA + fmaf(K1.y, y[jj], ty[jj]);
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const float det = fmaf(K0.z, z[q], detB), L = LB + lz[q];
                const float v = fminf(det, fmaf(-thr, (L * L) * L, det * det));
                s[jj][q] = r == 0 ? v : fminf(s[jj][q], v);
            }
        }
    }
    unsigned alive = 0;
#pragma unroll
    for (int jj = 0; jj < 2; ++jj)
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if (s[jj][q] > 0.f) alive |= 1u << (jj * 8 + q);
    return alive;
}

// Ring key with the tets spread over the lanes and a warp minimum of the per-tet keys (det if
// negative, else det^2 / L^3): the minimum needs no fixed order, so this costs one tet per lane
// and five shuffles. It can differ from tet_key1 in the last bit when two tets' fractions are
// within rounding of each other, so only the learned search, whose moves are judged by keys of
// this same function, uses it.
__device__ __forceinline__ float tet_key_min(const float4* __restrict__ co, int k, float x, float y, float z, int lane) {
    float m = FLT_MAX;
    for (int t = lane; t < k; t += 32) m = fminf(m, tet_piece_key(co, t, x, y, z));
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fminf(m, __shfl_xor_sync(FULL, m, o));
    return m;
}

// Setup of one tet vertex shared by the plain and the learned search: per-axis extent of the
// ring (DMOTetImplCub.h:54-64), the exact power-of-two scale 2^ex and the element coefficients
// in shared memory. Returns false when the ring is degenerate (the vertex is left alone).
// KEEP: rings of up to 32 tets (all of a Kuhn cube's) keep their lane's corners in registers
// between the extent and the coefficients; otherwise the corners are loaded again.
template <bool KEEP>
__device__ __forceinline__ bool tet_setup(const float4* __restrict__ pos, const int4* __restrict__ hf, int b, int k,
                                          float4 c0, int lane, float4* co, float& sx, float& sy, float& sz, int& ex) {
    float mdx = 0.f, mdy = 0.f, mdz = 0.f;
    const bool one = KEEP && k <= 32;
    float4 qa = c0, qb = c0, qc = c0;
    if (one) {
        if (lane < k) {
            const int4 h = hf[b + lane];
            qa = pos[h.x]; qb = pos[h.y]; qc = pos[h.z];
        }
        mdx = fmaxf(fabsf(qa.x - c0.x), fmaxf(fabsf(qb.x - c0.x), fabsf(qc.x - c0.x)));
        mdy = fmaxf(fabsf(qa.y - c0.y), fmaxf(fabsf(qb.y - c0.y), fabsf(qc.y - c0.y)));
        mdz = fmaxf(fabsf(qa.z - c0.z), fmaxf(fabsf(qb.z - c0.z), fabsf(qc.z - c0.z)));
    } else {
        for (int t = lane; t < k; t += 32) {
            const int4 h = hf[b + t];
            const float4 pa = pos[h.x], pb = pos[h.y], pc = pos[h.z];
            mdx = fmaxf(mdx, fabsf(pa.x - c0.x)); mdy = fmaxf(mdy, fabsf(pa.y - c0.y)); mdz = fmaxf(mdz, fabsf(pa.z - c0.z));
            mdx = fmaxf(mdx, fabsf(pb.x - c0.x)); mdy = fmaxf(mdy, fabsf(pb.y - c0.y)); mdz = fmaxf(mdz, fabsf(pb.z - c0.z));
            mdx = fmaxf(mdx, fabsf(pc.x - c0.x)); mdy = fmaxf(mdy, fabsf(pc.y - c0.y)); mdz = fmaxf(mdz, fabsf(pc.z - c0.z));
        }
    }
    mdx = warp_max(mdx); mdy = warp_max(mdy); mdz = warp_max(mdz);
    const float mm = fmaxf(mdx, fmaxf(mdy, mdz));
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return false;
    (void)frexpf(mm, &ex);
    const float p = exp2_exact(-ex);
    for (int t = lane; t < k; t += 32) {
        float4 pa = qa, pb = qb, pc = qc;
        if (!one) {
            const int4 h = hf[b + t];
            pa = pos[h.x]; pb = pos[h.y]; pc = pos[h.z];
        }
        float4 K0, K1;
        tet_coeffs(scale2(pa.x - c0.x, p, -ex), scale2(pa.y - c0.y, p, -ex), scale2(pa.z - c0.z, p, -ex),
                   scale2(pb.x - c0.x, p, -ex), scale2(pb.y - c0.y, p, -ex), scale2(pb.z - c0.z, p, -ex),
                   scale2(pc.x - c0.x, p, -ex), scale2(pc.y - c0.y, p, -ex), scale2(pc.z - c0.z, p, -ex), K0, K1);
        co[2 * t] = K0;
        co[2 * t + 1] = K1;
    }
    __syncwarp();
    sx = scale2(mdx, p, -ex); sy = scale2(mdy, p, -ex); sz = scale2(mdz, p, -ex);
    return true;
}

// position c0 + (dx, dy, dz) 2^ex of a move found in scaled local coordinates
__device__ __forceinline__ float4 tet_unscale(float4 c0, float dx, float dy, float dz, int ex) {
    const float p = exp2_exact(ex);
    return make_float4(c0.x + scale2(dx, p, ex), c0.y + scale2(dy, p, ex), c0.z + scale2(dz, p, ex), c0.w);
}

// The plain hierarchical search (DMOTetImplCub.h:66-136) from the local origin: depth levels
// of 8 x 8 x 8 candidates, moving on strict improvement of the ring key qLast. Returns whether
// the vertex moved; (dx, dy, dz) is the new position in scaled local coordinates.
__device__ __forceinline__ bool tet_plain_search(const float4* __restrict__ co, int* __restrict__ list, int k, float sx,
                                                 float sy, float sz, float grid_scale, int depth, int lane, float qLast,
                                                 float& dx, float& dy, float& dz) {
    const int ci = lane & 7, cj = lane >> 3;
    const float oi = grid_offset(ci), oj0 = grid_offset(cj), oj1 = grid_offset(cj + 4);
    dx = 0.f; dy = 0.f; dz = 0.f;
    bool moved = false;
    float ds = grid_scale;
    for (int level = 0; level < depth; ++level) {
        const float Sx = ds * sx, Sy = ds * sy, Sz = ds * sz;
        const float x = fmaf(oi, Sx, dx);
        const float y[2] = { fmaf(oj0, Sy, dy), fmaf(oj1, Sy, dy) };
        float z[NQ], tz[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) { z[q] = fmaf(grid_offset(q), Sz, dz); tz[q] = (3.0f * z[q]) * z[q]; }
        float bk = -FLT_MAX;
        int bi = 1 << 30;
        // filter: candidates already below qLast over the centre's critical tets are dropped
        int crit[TET_CRIT];
        tet_critical(co, k, dx, dy, dz, lane, crit);
        const float thr = qLast - (fabsf(qLast) * 0x1p-14f + 1e-37f);
        const unsigned alive = thr > 0.f ? tet_filter_pos(co, crit, min(TET_CRIT, k), x, y, z, tz, thr)
                                         : tet_filter(co, crit, min(TET_CRIT, k), x, y, z, tz, thr);
        const int cnt = __popc(alive);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int n = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += n;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        if (total > TET_LIST) {
#if TET_SPLIT_Y
            tet_lane_best<1>(co, k, x, &y[0], z, tz, ci, cj, 0, bk, bi);
            tet_lane_best<1>(co, k, x, &y[1], z, tz, ci, cj, 1, bk, bi);
#else
            tet_lane_best<2>(co, k, x, y, z, tz, ci, cj, 0, bk, bi);
#endif
        } else if (total > 0) {
            int at = incl - cnt;
            for (unsigned a = alive; a; a &= a - 1) {
                const int bit = __ffs(a) - 1;
                list[at++] = ci + 8 * (cj + 4 * (bit >> 3)) + 64 * (bit & 7);
            }
            __syncwarp();
            for (int j = lane; j < total; j += 32) {
                const int idx = list[j];
                const float key = tet_key1(co, k, fmaf(grid_offset(idx & 7), Sx, dx),
                                           fmaf(grid_offset((idx >> 3) & 7), Sy, dy), fmaf(grid_offset(idx >> 6), Sz, dz));
                if (key > bk || (key == bk && idx < bi)) { bk = key; bi = idx; }
            }
            __syncwarp();
        }
        warp_argmax(bk, bi);
        if (bi < NQ * NQ * NQ && qLast < bk) {
            const float nx = fmaf(grid_offset(bi & 7), Sx, dx);
            const float ny = fmaf(grid_offset((bi >> 3) & 7), Sy, dy);
            const float nz = fmaf(grid_offset(bi >> 6), Sz, dz);
            dx = nx; dy = ny; dz = nz;
            qLast = bk;
            moved = true;
        }
        ds = ds * (2.0f / 7.0f);
    }
    return moved;
}

// Active set (optional, dirty != null): a vertex whose last search found no improvement and
// none of whose ring vertices moved since is skipped -- the search would see the same ring and
// return the same "no move", so skipping changes no result. A search that finds nothing clears
// the vertex's flag; a move sets the flags of its ring vertices (adjacent vertices are never in
// the same colour class, so no flag a launch reads is written by that launch).
__device__ __forceinline__ void tet_mark_ring(const int4* __restrict__ hf, int b, int k, int lane,
                                              uint8_t* __restrict__ dirty) {
    for (int t = lane; t < k; t += 32) {
        const int4 h = hf[b + t];
        dirty[h.x] = 1; dirty[h.y] = 1; dirty[h.z] = 1;
    }
}

__global__ void __launch_bounds__(TET_WARPS * 32, TET_MIN_BLOCKS)
k_dmo_tet(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hf,
          int v0, int v1, float grid_scale, int depth, int maxk, uint8_t* __restrict__ dirty,
          unsigned long long* __restrict__ skipped) {
    extern __shared__ float4 smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int v = v0 + blockIdx.x * TET_WARPS + w;
    if (v >= v1) return;
    if (dirty && !dirty[v]) {
        if (lane == 0 && skipped) atomicAdd(skipped, 1ull);
        return;
    }
    float4* co = smem + (size_t)w * maxk * 2;
    int* list = reinterpret_cast<int*>(smem + (size_t)TET_WARPS * maxk * 2) + w * TET_LIST;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = pos[v];
    float sx, sy, sz;
    int ex;
    if (!tet_setup<true>(pos, hf, b, k, c0, lane, co, sx, sy, sz, ex)) return;
    const float qLast = tet_key_origin(co, k);
    float dx, dy, dz;
    const bool moved = tet_plain_search(co, list, k, sx, sy, sz, grid_scale, depth, lane, qLast, dx, dy, dz);
    if (moved && lane == 0) pos[v] = tet_unscale(c0, dx, dy, dz, ex);
    if (dirty) {
        if (moved) tet_mark_ring(hf, b, k, lane, dirty);
        else if (lane == 0) dirty[v] = 0;
    }
}

// The plain search over a list of vertices of one colour class (the learned mode's fallback):
// warps stride over list[0 .. count[0]). The last warp to finish sets the queue back to empty
// (count[0] = 0; count[1] counts the finished warps), so the next class's learned search
// appends to an empty queue without a separate reset launch.
#ifndef TET_LIST_MIN_BLOCKS
#define TET_LIST_MIN_BLOCKS 4   // 128 registers: four blocks per SM (164 unconstrained, three blocks)
#endif
__global__ void __launch_bounds__(TET_WARPS * 32, TET_LIST_MIN_BLOCKS)
k_dmo_tet_list(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hf,
               const int* __restrict__ list, int* __restrict__ count, float grid_scale, int depth, int maxk,
               uint8_t* __restrict__ dirty, unsigned long long* __restrict__ moved_count) {
    extern __shared__ float4 smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float4* co = smem + (size_t)w * maxk * 2;
    int* slist = reinterpret_cast<int*>(smem + (size_t)TET_WARPS * maxk * 2) + w * TET_LIST;
    const int n = *count;
    for (int idx = blockIdx.x * TET_WARPS + w; idx < n; idx += gridDim.x * TET_WARPS) {
        const int v = list[idx];
        const int b = rowptr[v], k = rowptr[v + 1] - b;
        if (k <= 0 || k > maxk) continue;
        const float4 c0 = pos[v];
        float sx, sy, sz;
        int ex;
        if (!tet_setup<true>(pos, hf, b, k, c0, lane, co, sx, sy, sz, ex)) continue;
        const float qLast = tet_key_origin(co, k);
        float dx, dy, dz;
        const bool moved = tet_plain_search(co, slist, k, sx, sy, sz, grid_scale, depth, lane, qLast, dx, dy, dz);
        if (moved && lane == 0) {
            pos[v] = tet_unscale(c0, dx, dy, dz, ex);
            atomicAdd(moved_count, 1ull);
        }
        if (dirty) {
            if (moved) tet_mark_ring(hf, b, k, lane, dirty);
            else if (lane == 0) dirty[v] = 0;
        }
        __syncwarp();
    }
    // every lane of this warp has read count[0]; the last warp of the grid resets the queue (a
    // warp count, not a block barrier: the warps of a block finish their strides apart)
    __syncwarp();
    if (lane == 0) {
        unsigned* done = reinterpret_cast<unsigned*>(count + 1);
        if (atomicAdd(done, 1u) == gridDim.x * TET_WARPS - 1) {
            count[0] = 0;
            *done = 0u;
        }
    }
}

// ---- learned proposal (tet) -------------------------------------------------------------------
// Distinct ring vertices of every vertex in [v0, v1), in first-occurrence order of its
// halfface row, at most 32 (the topology is fixed, so this runs once per optimiser):
// nb [(v - v0) * 32 + a], nbn [v - v0].
__global__ void k_tet_neighbours(const int* __restrict__ rowptr, const int4* __restrict__ hf, int v0, int v1,
                                 int* __restrict__ nb, int* __restrict__ nbn) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v1 - v0; i += gridDim.x * blockDim.x) {
        const int v = v0 + i;
        const int b = rowptr[v], k = rowptr[v + 1] - b;
        int* out = nb + (size_t)i * 32;
        int n = 0;
        for (int t = 0; t < k; ++t) {
            const int4 h = hf[b + t];
            const int u3[3] = { h.x, h.y, h.z };
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                bool seen = false;
                for (int a = 0; a < n; ++a) seen |= out[a] == u3[j];
                if (!seen && n < 32) out[n++] = u3[j];
            }
        }
        nbn[i] = n;
    }
}

// Features of the vertices [v0, v1): the ring vertices nb (in first-occurrence order of the
// halfface row, at most 32) relative to the vertex and divided by the ring's largest
// per-axis extent mm, zero padded to 96 values; FP32 rows and / or BF16 packed rows of the
// network's input operand. scale[i] = mm, old[i] = the vertex position. nb / nbn index the
// range relative to nb_base (the first vertex of the table).
__global__ void k_tet_features(const float4* __restrict__ pos, int v0, int v1, const int* __restrict__ nb,
                               const int* __restrict__ nbn, int nb_base, float* __restrict__ feats,
                               uint8_t* __restrict__ packed, float* __restrict__ scale, float4* __restrict__ old) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v1 - v0; i += gridDim.x * blockDim.x) {
        const int v = v0 + i;
        const float4 c0 = pos[v];
        const int* list = nb + (size_t)(v - nb_base) * 32;
        const int n = nbn[v - nb_base];
        // each ring vertex loaded once; the 96 inputs stay in registers (fully unrolled)
        float f[96];
        float mm = 0.f;
#pragma unroll
        for (int a = 0; a < 32; ++a) {
            float dx = 0.f, dy = 0.f, dz = 0.f;
            if (a < n) {
                const float4 q = pos[list[a]];
                dx = q.x - c0.x; dy = q.y - c0.y; dz = q.z - c0.z;
                mm = fmaxf(mm, fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))));
            }
            f[3 * a] = dx; f[3 * a + 1] = dy; f[3 * a + 2] = dz;
        }
        const float inv = mm > 0.f ? 1.f / mm : 0.f;
#pragma unroll
        for (int c = 0; c < 96; ++c) f[c] = f[c] * inv;
        if (scale) scale[i] = mm;
        if (old) old[i] = c0;
        if (feats) {
            float4* o = reinterpret_cast<float4*>(feats + (size_t)i * 96);
#pragma unroll
            for (int g = 0; g < 24; ++g) o[g] = make_float4(f[4 * g], f[4 * g + 1], f[4 * g + 2], f[4 * g + 3]);
        }
        if (packed) {
#pragma unroll
            for (int g = 0; g < 12; ++g) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) h[e] = __float2bfloat16_rn(f[8 * g + e]);
                *reinterpret_cast<uint4*>(packed + learned_pk_off(i, 8 * g)) = *reinterpret_cast<const uint4*>(h);
            }
        }
    }
}

// training targets of the vertices [v0, v1) after a plain colour launch: the displacement the
// search chose, in units of the ring extent
__global__ void k_tet_targets(const float4* __restrict__ pos, int v0, int v1, const float* __restrict__ scale,
                              const float4* __restrict__ old, float* __restrict__ targets) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v1 - v0; i += gridDim.x * blockDim.x) {
        const float4 p = pos[v0 + i], o = old[i];
        const float inv = scale[i] > 0.f ? 1.f / scale[i] : 0.f;
        targets[(size_t)i * 3 + 0] = (p.x - o.x) * inv;
        targets[(size_t)i * 3 + 1] = (p.y - o.y) * inv;
        targets[(size_t)i * 3 + 2] = (p.z - o.z) * inv;
    }
}

// offsets of the reduced grid with n points per axis: (n - 1 - 2i) / (n - 1)
// The 4^3 reduced search ranks its candidates by the LEARNED_CRIT tets of smallest exact key
// at the level's centre (ties to the lower tet), then judges the best-ranked one by its full
// ring key: within the small grid around the proposal the ring minimum of a candidate almost
// always sits in one of those tets, and a third of the ring costs a third of the search.
constexpr int LEARNED_CRIT = 8;

__device__ __forceinline__ void learned_critical(const float4* __restrict__ co, int k, float x, float y, float z,
                                                 int lane, int (&crit)[LEARNED_CRIT]) {
    if (k <= 32) {
        unsigned mine = lane < k ? tet_order_key(tet_piece_key(co, lane, x, y, z), lane) : 0xffffffffu;
#pragma unroll
        for (int r = 0; r < LEARNED_CRIT; ++r) {
            const unsigned m = __reduce_min_sync(FULL, mine);
            const int t = (int)(m & 31u);
            crit[r] = t < k ? t : 0;
            if (lane == t) mine = 0xffffffffu;
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < LEARNED_CRIT; ++r) {
        unsigned best = 0xffffffffu;
        int bt = 0;
        for (int t = lane; t < k; t += 32) {
            bool used = false;
#pragma unroll
            for (int q = 0; q < r; ++q) used |= (crit[q] == t);
            if (used) continue;
            const unsigned kt = tet_order_key(tet_piece_key(co, t, x, y, z), t & 31);
            if (kt < best || (kt == best && t < bt)) { best = kt; bt = t; }
        }
        const unsigned m = __reduce_min_sync(FULL, best);
        const unsigned tt = __reduce_min_sync(FULL, best == m ? (unsigned)bt : 0xffffffffu);
        crit[r] = tt < (unsigned)k ? (int)tt : 0;
    }
}

__device__ __forceinline__ float reduced_offset(int i, int n) { return (float)(n - 1 - 2 * i) / (float)(n - 1); }

// Learned search: the network's displacement y (units of mm) centres a reduced grid of
// rn^3 candidates per level, rdepth levels, half-extent starting at the plain search's second
// level (grid_scale * 2/7 of the ring extent) and shrinking by 2/(rn-1); the proposal itself is
// a candidate too. The vertex moves when the best of them strictly raises its ring minimum;
// otherwise the full plain search runs (fallback), so every move is one plain DMO could
// accept and the minimum quality never decreases. counters: [0] reduced accepted,
// [1] fallbacks, [2] fallbacks that moved, [3] skipped by the active set. rscale: first
// reduced half-extent in units of grid_scale x the per-axis ring extent.
// eight blocks per SM (64 registers, 16 bytes of spills) with the ring corners kept through the
// setup: 2.3 % less time per learned iteration than seven blocks at 72 registers without
#ifndef TET_LEARNED_MIN_BLOCKS
#define TET_LEARNED_MIN_BLOCKS 8
#endif
#ifndef TET_LEARNED_KEEP
#define TET_LEARNED_KEEP true
#endif
__global__ void __launch_bounds__(TET_WARPS * 32, TET_LEARNED_MIN_BLOCKS)
k_dmo_tet_learned(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hf, int v0,
                  int v1, float grid_scale, int maxk, const float* __restrict__ Y, int ldy, int rn, int rdepth,
                  float rscale, unsigned long long* __restrict__ counters, uint8_t* __restrict__ dirty,
                  int* __restrict__ fb_list, int* __restrict__ fb_count) {
    extern __shared__ float4 smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int v = v0 + blockIdx.x * TET_WARPS + w;
    if (v >= v1) return;
    if (dirty && !dirty[v]) {
        if (lane == 0) atomicAdd(&counters[3], 1ull);
        return;
    }
    float4* co = smem + (size_t)w * maxk * 2;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = pos[v];
    float sx, sy, sz;
    int ex;
    if (!tet_setup<TET_LEARNED_KEEP>(pos, hf, b, k, c0, lane, co, sx, sy, sz, ex)) return;
    const float q0 = tet_key_min(co, k, 0.f, 0.f, 0.f, lane);
    // proposal in scaled local coordinates (the features were divided by mm = max(sx, sy, sz) 2^ex)
    const float mms = fmaxf(sx, fmaxf(sy, sz));
    const float* y = Y + (size_t)(v - v0) * ldy;
    float px = y[0] * mms, py = y[1] * mms, pz = y[2] * mms;
    const float bx = grid_scale * sx, by = grid_scale * sy, bz = grid_scale * sz;
    const bool have = isfinite(px) && isfinite(py) && isfinite(pz);
    float best = -FLT_MAX, cx = 0.f, cy = 0.f, cz = 0.f;
    if (have) {
        px = fminf(fmaxf(px, -bx), bx); py = fminf(fmaxf(py, -by), by); pz = fminf(fmaxf(pz, -bz), bz);
        best = tet_key_min(co, k, px, py, pz, lane);
        cx = px; cy = py; cz = pz;
        float rx = grid_scale * rscale * sx, ry = grid_scale * rscale * sy, rz = grid_scale * rscale * sz;
        const int nc = rn * rn * rn;
        for (int level = 0; level < rdepth; ++level) {
            float bk = -FLT_MAX;
            int bi = 1 << 30;
            if (rn == 4) {
                // 64 candidates, index ix + 4 iy + 16 iz: lane (ix, iy, iz0) also takes iz0 + 2,
                // sharing the x and y parts of every tet; offsets (3 - 2i) / 3; ranked over the
                // critical tets of the centre
                const int ix = lane & 3, iy = (lane >> 2) & 3, iz0 = lane >> 4;
                const float o4[4] = { 1.0f, 1.0f / 3.0f, -1.0f / 3.0f, -1.0f };
                const float x = fmaf(o4[ix], rx, cx);
                const float yy = fmaf(o4[iy], ry, cy);
                const float z0 = fmaf(o4[iz0], rz, cz), z1 = fmaf(o4[iz0 + 2], rz, cz);
                const float tx = (3.0f * x) * x, ty = (3.0f * yy) * yy;
                const float tz0 = (3.0f * z0) * z0, tz1 = (3.0f * z1) * z1;
                float N0 = 0.f, D0 = 1.f, m0 = 0.f, N1 = 0.f, D1 = 1.f, m1 = 0.f;
                int crit[LEARNED_CRIT];
                learned_critical(co, k, cx, cy, cz, lane, crit);
                const int nt = min(LEARNED_CRIT, k);
#pragma unroll
                for (int r = 0; r < LEARNED_CRIT; ++r) {
                    if (r >= nt) break;
                    const int t = crit[r];
                    const float4 K0 = co[2 * t], K1 = co[2 * t + 1];
                    const float detB = fmaf(K0.y, yy, fmaf(K0.x, x, K0.w));
                    const float LB = (K1.w + fmaf(K1.x, x, tx)) + fmaf(K1.y, yy, ty);
                    const float d0 = fmaf(K0.z, z0, detB), L0 = LB + fmaf(K1.z, z0, tz0);
                    const float d1 = fmaf(K0.z, z1, detB), L1 = LB + fmaf(K1.z, z1, tz1);
                    const float n0 = d0 * d0, e0 = (L0 * L0) * L0, n1 = d1 * d1, e1 = (L1 * L1) * L1;
                    if (r == 0) { N0 = n0; D0 = e0; m0 = d0; N1 = n1; D1 = e1; m1 = d1; continue; }
                    if (n0 * D0 < N0 * e0) { N0 = n0; D0 = e0; }
                    if (n1 * D1 < N1 * e1) { N1 = n1; D1 = e1; }
                    m0 = fminf(m0, d0); m1 = fminf(m1, d1);
                }
                const float k0 = m0 < 0.f ? m0 : N0 / D0, k1 = m1 < 0.f ? m1 : N1 / D1;
                bk = k0; bi = lane;
                if (k1 > bk) { bk = k1; bi = lane + 32; }
            } else {
                for (int c = lane; c < nc; c += 32) {
                    const int ix = c % rn, iy = (c / rn) % rn, iz = c / (rn * rn);
                    const float x = fmaf(reduced_offset(ix, rn), rx, cx);
                    const float yy = fmaf(reduced_offset(iy, rn), ry, cy);
                    const float z = fmaf(reduced_offset(iz, rn), rz, cz);
                    const float key = tet_key1(co, k, x, yy, z);
                    if (key > bk || (key == bk && c < bi)) { bk = key; bi = c; }
                }
            }
            warp_argmax(bk, bi);
            if (rn == 4 && bi < nc && bk > best) {
                // the best-ranked candidate is judged by its full ring key
                const int ix = bi % rn, iy = (bi / rn) % rn, iz = bi / (rn * rn);
                bk = tet_key_min(co, k, fmaf(reduced_offset(ix, rn), rx, cx), fmaf(reduced_offset(iy, rn), ry, cy),
                                 fmaf(reduced_offset(iz, rn), rz, cz), lane);
            }
            if (bi < nc && bk > best) {
                const int ix = bi % rn, iy = (bi / rn) % rn, iz = bi / (rn * rn);
                const float nx = fmaf(reduced_offset(ix, rn), rx, cx);
                const float ny = fmaf(reduced_offset(iy, rn), ry, cy);
                const float nz = fmaf(reduced_offset(iz, rn), rz, cz);
                cx = nx; cy = ny; cz = nz;
                best = bk;
            }
            const float sh = 2.0f / (float)(rn - 1);
            rx *= sh; ry *= sh; rz *= sh;
        }
    }
    if (have && best > q0) {
        if (lane == 0) {
            pos[v] = tet_unscale(c0, cx, cy, cz, ex);
            atomicAdd(&counters[0], 1ull);
        }
        if (dirty) tet_mark_ring(hf, b, k, lane, dirty);
        return;
    }
    // the proposal did not raise the ring minimum: queue the vertex for the plain search
    if (lane == 0) {
        fb_list[atomicAdd(fb_count, 1)] = v;
        atomicAdd(&counters[1], 1ull);
    }
}


// ---- hexahedra ------------------------------------------------------------------------------------
// k_optimizeHierarchicalInnerHex<128> (dmo/DMOHexImplCub.h:21-137) with shapeMetricHex
// (dmo/DMOQualityHex.h:54-71). With the candidate p as corner 0 of a halfhex, sub-tets 1, 2, 3
// and 6 of the metric do not depend on p, and sub-tets 0, 4, 5, 7, 8 have a determinant affine
// in p and a Frobenius term quadratic in p; each halfhex is staged as 43 coefficients (the
// constant part's key and 5 x {g, c, m, C}). min_j cbrt(s^2) / A is compared through s^2 / A^3
// as a fraction. The reference block's 128 threads of 4 candidates, whose maxima carry across
// levels, are kept as one block of 128 threads per vertex: thread t takes candidates
// 4t .. 4t+3 (x = 4 (t & 1) .. +3, y = (t >> 1) & 7, z = t >> 4). (The colour classes of a hex
// mesh hold ~600-1,200 vertices: one warp per vertex left ~8 warps per SM.)
constexpr int HEX_THREADS = 128;
constexpr int HEX_MAX_RING = 64;

__global__ void __launch_bounds__(HEX_THREADS)
k_dmo_hex(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ hh, int v0,
          float grid_scale, int depth, int maxk) {
    extern __shared__ float4 smem[];
    __shared__ float red[6][HEX_THREADS / 32];
    __shared__ float s_k[HEX_THREADS / 32];
    __shared__ int s_i[HEX_THREADS / 32];
    __shared__ float s_win[3];
    __shared__ float s_qlast;
    __shared__ int s_czero;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int v = v0 + blockIdx.x;
    float* co = reinterpret_cast<float*>(smem);
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = pos[v];
    // per-axis largest (scale) and smallest (grid extent, DMOHexImplCub.h:49-68) ring distance
    float mx0 = 0.f, mx1 = 0.f, mx2 = 0.f, mn0 = FLT_MAX, mn1 = FLT_MAX, mn2 = FLT_MAX;
    for (int idx = t; idx < 7 * k; idx += HEX_THREADS) {
        const int h = idx / 7, c = idx % 7;
        const int4 q = hh[2 * (b + h) + (c >> 2)];
        const int cc = c & 3;
        const int u = cc == 0 ? q.x : (cc == 1 ? q.y : (cc == 2 ? q.z : q.w));
        const float4 p = pos[u];
        const float d0 = fabsf(p.x - c0.x), d1 = fabsf(p.y - c0.y), d2 = fabsf(p.z - c0.z);
        mx0 = fmaxf(mx0, d0); mx1 = fmaxf(mx1, d1); mx2 = fmaxf(mx2, d2);
        mn0 = fminf(mn0, d0); mn1 = fminf(mn1, d1); mn2 = fminf(mn2, d2);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        mx0 = fmaxf(mx0, __shfl_xor_sync(FULL, mx0, o)); mx1 = fmaxf(mx1, __shfl_xor_sync(FULL, mx1, o));
        mx2 = fmaxf(mx2, __shfl_xor_sync(FULL, mx2, o)); mn0 = fminf(mn0, __shfl_xor_sync(FULL, mn0, o));
        mn1 = fminf(mn1, __shfl_xor_sync(FULL, mn1, o)); mn2 = fminf(mn2, __shfl_xor_sync(FULL, mn2, o));
    }
    if (lane == 0) { red[0][w] = mx0; red[1][w] = mx1; red[2][w] = mx2; red[3][w] = mn0; red[4][w] = mn1; red[5][w] = mn2; }
    if (t == 0) s_czero = 0;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < HEX_THREADS / 32; ++i) {
        mx0 = fmaxf(mx0, red[0][i]); mx1 = fmaxf(mx1, red[1][i]); mx2 = fmaxf(mx2, red[2][i]);
        mn0 = fminf(mn0, red[3][i]); mn1 = fminf(mn1, red[4][i]); mn2 = fminf(mn2, red[5][i]);
    }
    const float mm = fmaxf(mx0, fmaxf(mx1, mx2));
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return;   // uniform over the block
    int ex;
    (void)frexpf(mm, &ex);
    const float p2 = exp2_exact(-ex);
    const float es = ldexpf(HEX_EPS, -3 * ex), ea = ldexpf(HEX_EPS, -2 * ex);
    for (int h = t; h < k; h += HEX_THREADS) {
        const int4 qa = hh[2 * (b + h)], qb = hh[2 * (b + h) + 1];
        const int us[7] = { qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z };
        float r[7][3];
#pragma unroll
        for (int c = 0; c < 7; ++c) {
            const float4 p = pos[us[c]];
            r[c][0] = scale2(p.x - c0.x, p2, -ex); r[c][1] = scale2(p.y - c0.y, p2, -ex); r[c][2] = scale2(p.z - c0.z, p2, -ex);
        }
        hex_coeffs(r, es, ea, co + HEX_CO * h);
        if (co[HEX_CO * h + 2] != 0.f) s_czero = 1;
    }
    __syncthreads();
    const float sx = scale2(mn0, p2, -ex), sy = scale2(mn1, p2, -ex), sz = scale2(mn2, p2, -ex);
    // ring-wide: any constant part zero makes every candidate's key zero
    const bool czero = s_czero != 0;
    const int ci = 4 * (t & 1), cj = (t >> 1) & 7, ck = t >> 4;
    float qMax = -FLT_MAX, pX = 0.f, pY = 0.f, pZ = 0.f;
    float dx = 0.f, dy = 0.f, dz = 0.f;
    float ds = grid_scale;
    float qWin = -FLT_MAX;
    for (int level = 0; level < depth; ++level) {
        const float Sx = ds * sx, Sy = ds * sy, Sz = ds * sz;
        // the key at the current position: one warp computes it while the others search
        if (w == 0) {
            const float q = hex_key1(co, k, dx, dy, dz, es, ea);
            if (lane == 0) s_qlast = q;
        }
        const float z = fmaf(grid_offset(ck), Sz, dz);
        const float y = fmaf(grid_offset(cj), Sy, dy);
        float x[4], t1x[4], t3x[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) { x[i] = fmaf(grid_offset(ci + i), Sx, dx); t1x[i] = x[i] * x[i]; t3x[i] = (3.f * x[i]) * x[i]; }
        const float t1z = z * z, t3z = (3.f * z) * z;
        const float t1y = y * y, t3y = (3.f * y) * y;
        float N[4], D[4];
        bool zr[4];
        {
            const float n0 = co[0], d0 = co[1];
#pragma unroll
            for (int i = 0; i < 4; ++i) { N[i] = n0; D[i] = d0; zr[i] = czero; }
        }
        for (int h = 0; h < k; ++h) {
            const float* c = co + HEX_CO * h;
            if (h > 0) {
                const float cn = c[0], cd = c[1];
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (cn * D[i] < N[i] * cd) { N[i] = cn; D[i] = cd; }
            }
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                const float* q = c + 3 + 8 * j;
                const bool a3 = (j == 1 || j == 4);
                const float sY = fmaf(q[1], y, fmaf(q[2], z, q[3]));
                const float aY = (q[7] + fmaf(q[6], z, a3 ? t3z : t1z)) + fmaf(q[5], y, a3 ? t3y : t1y);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float sd = fmaf(q[0], x[i], sY);
                    const float A = aY + fmaf(q[4], x[i], a3 ? t3x[i] : t1x[i]);
                    if (sd < es || A < ea) { zr[i] = true; continue; }
                    const float num = sd * sd, den = (A * A) * A;
                    if (num * D[i] < N[i] * den) { N[i] = num; D[i] = den; }
                }
            }
        }
        // the thread's maximum carries across levels (candidates in index order, strict >)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float key = zr[i] ? 0.f : N[i] / D[i];
            if (key > qMax) { qMax = key; pX = x[i]; pY = y; pZ = z; }
        }
        // block arg-max, the lowest thread on ties
        float bk = qMax;
        int bi = t;
        warp_argmax(bk, bi);
        if (lane == 0) { s_k[w] = bk; s_i[w] = bi; }
        __syncthreads();
        bk = s_k[0]; bi = s_i[0];
#pragma unroll
        for (int i = 1; i < HEX_THREADS / 32; ++i)
            if (s_k[i] > bk || (s_k[i] == bk && s_i[i] < bi)) { bk = s_k[i]; bi = s_i[i]; }
        if (t == bi) { s_win[0] = pX; s_win[1] = pY; s_win[2] = pZ; }
        __syncthreads();
        if (s_qlast < bk) { dx = s_win[0]; dy = s_win[1]; dz = s_win[2]; }
        qWin = bk;
        ds = ds * (2.0f / 7.0f);
        __syncthreads();   // s_k / s_win are rewritten by the next level
    }
    if (t == 0 && hex_key1(co, k, 0.f, 0.f, 0.f, es, ea) < qWin) pos[v] = tet_unscale(c0, dx, dy, dz, ex);
}

// ---- flat triangles ---------------------------------------------------------------------------
__device__ __forceinline__ float tri_key(const float4* co, int k, float x, float y) {
    const float tx = (2.0f * x) * x, ty = (2.0f * y) * y;
    float N = 0.f, D = 1.f, am = 0.f;
    for (int t = 0; t < k; ++t) {
        const float4 c0 = co[2 * t], c1 = co[2 * t + 1];
        const float A = fmaf(c0.y, y, fmaf(c0.x, x, c0.z));
        const float L = (c0.w + fmaf(c1.x, x, tx)) + fmaf(c1.y, y, ty);
        if (t == 0) { N = A; D = L; am = A; continue; }
        if (A * D < N * L) { N = A; D = L; }
        am = fminf(am, A);
    }
    return am < 0.f ? am : N / D;
}

__global__ void __launch_bounds__(TRI_WARPS * 32)
k_dmo_tri2d(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he,
            int v0, int v1, float grid_scale, int depth, int maxk) {
    extern __shared__ float4 smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int v = v0 + blockIdx.x * TRI_WARPS + w;
    if (v >= v1) return;
    float4* co = smem + (size_t)w * maxk * 2;
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = pos[v];
    float mdx = 0.f, mdy = 0.f;
    for (int t = lane; t < k; t += 32) {
        const float4 p = pos[he[b + t].x];
        mdx = fmaxf(mdx, fabsf(p.x - c0.x));
        mdy = fmaxf(mdy, fabsf(p.y - c0.y));
    }
    mdx = warp_max(mdx); mdy = warp_max(mdy);
    const float mm = fmaxf(mdx, mdy);
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return;
    int ex;
    (void)frexpf(mm, &ex);
    const float p = exp2_exact(-ex);
    for (int t = lane; t < k; t += 32) {
        const float4 pa = pos[he[b + t].x];
        const float4 pb = pos[he[b + (t + 1 == k ? 0 : t + 1)].x];
        const float ax = scale2(pa.x - c0.x, p, -ex), ay = scale2(pa.y - c0.y, p, -ex);
        const float bx = scale2(pb.x - c0.x, p, -ex), by = scale2(pb.y - c0.y, p, -ex);
        const float ux = bx - ax, uy = by - ay;
        const float C = ((ax * ax + ay * ay) + (bx * bx + by * by)) + (ux * ux + uy * uy);
        co[2 * t] = make_float4(-uy, ux, ax * uy - ay * ux, C);
        co[2 * t + 1] = make_float4(-2.0f * (ax + bx), -2.0f * (ay + by), 0.f, 0.f);
    }
    __syncwarp();
    const float sx = scale2(mdx, p, -ex), sy = scale2(mdy, p, -ex);
    const int i1 = lane >> 3, j1 = lane & 7;
    const float o1 = grid_offset(i1), o2 = grid_offset(i1 + 4), oj = grid_offset(j1);
    float dx = 0.f, dy = 0.f;
    const float qOld = tri_key(co, k, 0.f, 0.f);
    float qLast = qOld, lastMax = -FLT_MAX;
    float ds = grid_scale;
    for (int level = 0; level < depth; ++level) {
        const float Sx = ds * sx, Sy = ds * sy;
        const float x1 = fmaf(o1, Sx, dx), x2 = fmaf(o2, Sx, dx), y = fmaf(oj, Sy, dy);
        const float q1 = tri_key(co, k, x1, y);
        const float q2 = tri_key(co, k, x2, y);
        float val = q1;
        if (q2 > q1) val = q2;
        const float selx = (q1 > q2) ? x1 : x2;
        float bv = val;
        int bl = lane;
        warp_argmax(bv, bl);
        if (qLast < bv) {
            dx = __shfl_sync(FULL, selx, bl);
            dy = __shfl_sync(FULL, y, bl);
            qLast = bv;
        }
        lastMax = bv;
        ds = ds * (2.0f / 7.0f);
    }
    if (qOld < lastMax && lane == 0)
        pos[v] = make_float4(c0.x + scale2(dx, exp2_exact(ex), ex), c0.y + scale2(dy, exp2_exact(ex), ex), c0.z, c0.w);
}

// ---- reference element metrics ---------------------------------------------------------------
// meanRatioMetricTet (dmo/DMOQualityTet.h:119-143)
__device__ __forceinline__ float q_tet(float4 p0, float4 p1, float4 p2, float4 p3) {
    const float e0x = p1.x - p0.x, e0y = p1.y - p0.y, e0z = p1.z - p0.z;
    const float e1x = p2.x - p0.x, e1y = p2.y - p0.y, e1z = p2.z - p0.z;
    const float e2x = p3.x - p0.x, e2y = p3.y - p0.y, e2z = p3.z - p0.z;
    const float cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
    const float volume = (1.f / 6.f) * ((e0x * cx + e0y * cy) + e0z * cz);
    if (volume < 0.f) return volume;
    const float mu = cbrtf(volume * volume);
    const float e3x = p2.x - p1.x, e3y = p2.y - p1.y, e3z = p2.z - p1.z;
    const float e4x = p3.x - p1.x, e4y = p3.y - p1.y, e4z = p3.z - p1.z;
    const float e5x = p3.x - p2.x, e5y = p3.y - p2.y, e5z = p3.z - p2.z;
    float l = 0.f;
    l += (e0x * e0x + e0y * e0y) + e0z * e0z;
    l += (e1x * e1x + e1y * e1y) + e1z * e1z;
    l += (e2x * e2x + e2y * e2y) + e2z * e2z;
    l += (e3x * e3x + e3y * e3y) + e3z * e3z;
    l += (e4x * e4x + e4y * e4y) + e4z * e4z;
    l += (e5x * e5x + e5y * e5y) + e5z * e5z;
    const float cbrtf9 = 2.0800838230519f;
    return ((12.f * cbrtf9) * mu) / l;
}

// meanRatioMetricTri2D (dmo/DMOQualityTri.h:243-257)
__device__ __forceinline__ float q_tri2d(float4 p0, float4 p1, float4 p2) {
    const float e0x = p1.x - p0.x, e0y = p1.y - p0.y;
    const float e1x = p2.x - p1.x, e1y = p2.y - p1.y;
    const float e2x = p0.x - p2.x, e2y = p0.y - p2.y;
    const float l = ((e0x * e0x + e0y * e0y) + (e1x * e1x + e1y * e1y)) + (e2x * e2x + e2y * e2y);
    const float area = e0x * e1y - e0y * e1x;
    if (area < 0.f) return area;
    return ((2.f * sqrtf(3.f)) * area) / l;
}

// meanRatioMetricTri(p) (dmo/DMOQualityTri.h:260-272), unsigned
__device__ __forceinline__ float q_tri3d(float4 p0, float4 p1, float4 p2) {
    const float e0x = p1.x - p0.x, e0y = p1.y - p0.y, e0z = p1.z - p0.z;
    const float e1x = p2.x - p0.x, e1y = p2.y - p0.y, e1z = p2.z - p0.z;
    const float e2x = p2.x - p1.x, e2y = p2.y - p1.y, e2z = p2.z - p1.z;
    const float l = (((e0x * e0x + e0y * e0y) + e0z * e0z) + ((e1x * e1x + e1y * e1y) + e1z * e1z)) +
                    ((e2x * e2x + e2y * e2y) + e2z * e2z);
    const float cx = e0y * e1z - e0z * e1y, cy = e0z * e1x - e0x * e1z, cz = e0x * e1y - e0y * e1x;
    return ((2.f * sqrtf(3.f)) * sqrtf((cx * cx + cy * cy) + cz * cz)) / l;
}

// meanRatioMetricQuad(p) (dmo/DMOQualityQuad.h:13-28): 2 (A1 + A2) / sum |e|^2
__device__ __forceinline__ float q_quad(float4 p0, float4 p1, float4 p2, float4 p3) {
    const float e0x = p1.x - p0.x, e0y = p1.y - p0.y, e0z = p1.z - p0.z;
    const float e1x = p2.x - p1.x, e1y = p2.y - p1.y, e1z = p2.z - p1.z;
    const float e2x = p3.x - p2.x, e2y = p3.y - p2.y, e2z = p3.z - p2.z;
    const float e3x = p0.x - p3.x, e3y = p0.y - p3.y, e3z = p0.z - p3.z;
    const float l = ((((e0x * e0x + e0y * e0y) + e0z * e0z) + ((e1x * e1x + e1y * e1y) + e1z * e1z)) +
                     ((e2x * e2x + e2y * e2y) + e2z * e2z)) + ((e3x * e3x + e3y * e3y) + e3z * e3z);
    const float m0x = -e0x, m0y = -e0y, m0z = -e0z, m2x = -e2x, m2y = -e2y, m2z = -e2z;
    const float c1x = e1y * m0z - e1z * m0y, c1y = e1z * m0x - e1x * m0z, c1z = e1x * m0y - e1y * m0x;
    const float c2x = e3y * m2z - e3z * m2y, c2y = e3z * m2x - e3x * m2z, c2z = e3x * m2y - e3y * m2x;
    const float a1 = sqrtf((c1x * c1x + c1y * c1y) + c1z * c1z);
    const float a2 = sqrtf((c2x * c2x + c2y * c2y) + c2z * c2z);
    return (2.f * (a1 + a2)) / l;
}

// meanRatioMetricQuad(p, n) with n = +z (dmo/DMOQualityQuad.h:30-50) for flat quads: -1 when a
// corner turns clockwise, else 2 (A1 + A2) / sum |e|^2 (the corner areas are the z components)
__device__ __forceinline__ float q_quad2d(float4 p0, float4 p1, float4 p2, float4 p3) {
    const float e0x = p1.x - p0.x, e0y = p1.y - p0.y, e1x = p2.x - p1.x, e1y = p2.y - p1.y;
    const float e2x = p3.x - p2.x, e2y = p3.y - p2.y, e3x = p0.x - p3.x, e3y = p0.y - p3.y;
    const float l = (((e0x * e0x + e0y * e0y) + (e1x * e1x + e1y * e1y)) + (e2x * e2x + e2y * e2y)) + (e3x * e3x + e3y * e3y);
    const float c1 = e1x * (-e0y) - e1y * (-e0x);
    const float c2 = e3x * (-e2y) - e3y * (-e2x);
    if (c1 < 0.f || c2 < 0.f) return -1.f;
    return (2.f * (c1 + c2)) / l;
}

// shapeMetricHex (dmo/DMOQualityHex.h:54-71) in the reference's operation order, with cbrtf
__device__ float q_hex(const float4* __restrict__ pos, const int* __restrict__ h) {
    float v[8][3];
#pragma unroll
    for (int c = 0; c < 8; ++c) { const float4 p = pos[h[c]]; v[c][0] = p.x; v[c][1] = p.y; v[c][2] = p.z; }
    const float* P[8] = { v[4], v[5], v[6], v[7], v[0], v[1], v[2], v[3] };
    float L[12][3], X[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        L[0][a] = P[1][a] - P[0][a]; L[4][a] = P[4][a] - P[0][a]; L[8][a] = P[5][a] - P[4][a];
        L[1][a] = P[2][a] - P[1][a]; L[5][a] = P[5][a] - P[1][a]; L[9][a] = P[6][a] - P[5][a];
        L[2][a] = P[3][a] - P[2][a]; L[6][a] = P[6][a] - P[2][a]; L[10][a] = P[7][a] - P[6][a];
        L[3][a] = P[3][a] - P[0][a]; L[7][a] = P[7][a] - P[3][a]; L[11][a] = P[7][a] - P[4][a];
        X[0][a] = (((P[1][a] - P[0][a]) + (P[2][a] - P[3][a])) + (P[5][a] - P[4][a])) + (P[6][a] - P[7][a]);
        X[1][a] = (((P[3][a] - P[0][a]) + (P[2][a] - P[1][a])) + (P[7][a] - P[4][a])) + (P[6][a] - P[5][a]);
        X[2][a] = (((P[4][a] - P[0][a]) + (P[5][a] - P[1][a])) + (P[6][a] - P[2][a])) + (P[7][a] - P[3][a]);
    }
    const int T[9][3] = { { 0, 3, 4 }, { 1, 0, 5 }, { 2, 1, 6 }, { 3, 2, 7 }, { 11, 8, 4 },
                          { 8, 9, 5 }, { 9, 10, 6 }, { 10, 11, 7 }, { 0, 1, 2 } };
    const int S[9][3] = { { 1, 1, 1 }, { 1, -1, 1 }, { 1, -1, 1 }, { -1, -1, 1 }, { 1, 1, -1 },
                          { -1, 1, -1 }, { -1, 1, -1 }, { -1, -1, -1 }, { 1, 1, 1 } };
    float ret = 1e30f;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        float e[3][3];
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float val = i == 8 ? X[T[i][j]][a] : L[T[i][j]][a];
                e[j][a] = S[i][j] < 0 ? -val : val;
            }
        float x[3];
        hcross(e[1], e[2], x);
        const float sj = hdot3(e[0], x);
        const float Aj = (hdot3(e[0], e[0]) + hdot3(e[1], e[1])) + hdot3(e[2], e[2]);
        if (sj < HEX_EPS || Aj < HEX_EPS) return 0.f;
        ret = fminf(ret, cbrtf(sj * sj) / Aj);
    }
    return 3.f * ret;
}

__device__ __forceinline__ float element_quality(const int* __restrict__ el, int kind, const float4* __restrict__ pos, long e) {
    if (kind == MK_HEX) return q_hex(pos, el + 8 * e);
    if (kind == MK_HEX_COND) {
        float v[8][3];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float4 p = pos[el[8 * e + c]];
            v[c][0] = p.x; v[c][1] = p.y; v[c][2] = p.z;
        }
        return hc_element_quality(v);
    }
    if (kind == MK_TET_MINA || kind == MK_TET_MAXA) {
        const int4 t = reinterpret_cast<const int4*>(el)[e];
        const float4 a = pos[t.x], b = pos[t.y], c = pos[t.z], d = pos[t.w];
        const float pa[3] = { a.x, a.y, a.z }, pb[3] = { b.x, b.y, b.z }, pc[3] = { c.x, c.y, c.z }, pd[3] = { d.x, d.y, d.z };
        return kind == MK_TET_MINA ? tet_angle<false>(pa, pb, pc, pd) : tet_angle<true>(pa, pb, pc, pd);
    }
    if (kind == MK_TRI2D_MINA || kind == MK_TRI2D_MAXA) {
        const int* t = el + 3 * e;
        const float4 a = pos[t[0]], b = pos[t[1]], c = pos[t[2]];
        return kind == MK_TRI2D_MINA ? tri2d_angle<false>(a.x, a.y, b.x, b.y, c.x, c.y)
                                     : tri2d_angle<true>(a.x, a.y, b.x, b.y, c.x, c.y);
    }
    if (kind == MK_TRI3D_MINA || kind == MK_TRI3D_MAXA) {
        const int* t = el + 3 * e;
        const float4 a = pos[t[0]], b = pos[t[1]], c = pos[t[2]];
        const float pa[3] = { a.x, a.y, a.z }, pb[3] = { b.x, b.y, b.z }, pc[3] = { c.x, c.y, c.z };
        return kind == MK_TRI3D_MINA ? tri3d_angle<false, false>(pa, pb, pc, 0.f, 0.f, 0.f)
                                     : tri3d_angle<true, false>(pa, pb, pc, 0.f, 0.f, 0.f);
    }
    if (kind == MK_TET) {
        const int4 t = reinterpret_cast<const int4*>(el)[e];
        return q_tet(pos[t.x], pos[t.y], pos[t.z], pos[t.w]);
    }
    if (kind == MK_QUAD || kind == MK_QUAD2D) {
        const int4 t = reinterpret_cast<const int4*>(el)[e];
        return kind == MK_QUAD ? q_quad(pos[t.x], pos[t.y], pos[t.z], pos[t.w]) : q_quad2d(pos[t.x], pos[t.y], pos[t.z], pos[t.w]);
    }
    if (kind == MK_QUAD_COND) {
        const int4 t = reinterpret_cast<const int4*>(el)[e];
        const float4 a = pos[t.x];
        return quad_cond<false>(a.x, a.y, a.z, pos[t.y], pos[t.z], pos[t.w], make_float3(0.f, 0.f, 0.f));
    }
    const int* t = el + 3 * e;
    if (kind == MK_TRI3D) return q_tri3d(pos[t[0]], pos[t[1]], pos[t[2]]);
    return q_tri2d(pos[t[0]], pos[t[1]], pos[t[2]]);
}

// the element loop is a chain of dependent loads (indices, then corners), bound by how many of
// them are in flight: four elements per thread, one resident grid (80 registers: 3 blocks of
// 256 threads per SM)
constexpr int QS_BLOCKS = 148 * 3;
constexpr int QS_THREADS = 256;
constexpr int QS_UNROLL = 4;

__global__ void __launch_bounds__(QS_THREADS)
k_quality_stats(const int* __restrict__ el, int kind, long nE, const float4* __restrict__ pos, IterStats* stats,
                int* iter, float* pmin, double* psum, int* pfail, unsigned* done, int check, int init) {
    __shared__ float smin[QS_THREADS / 32];
    __shared__ double ssum[QS_THREADS / 32];
    __shared__ int sfail[QS_THREADS / 32];
    __shared__ bool last;
    const int it = *iter;
    const float lastMin = init ? -FLT_MAX : stats[it].min_q;
    const float tol = 1e-6f * fmaxf(fabsf(lastMin), 1e-30f);
    float mn = FLT_MAX;
    double sm = 0.0;
    int fl = 0;
    const long st = (long)QS_BLOCKS * QS_THREADS;
    long e = (long)blockIdx.x * QS_THREADS + threadIdx.x;
    for (; e + (QS_UNROLL - 1) * st < nE; e += QS_UNROLL * st) {
        float q[QS_UNROLL];
#pragma unroll
        for (int j = 0; j < QS_UNROLL; ++j) q[j] = element_quality(el, kind, pos, e + j * st);
#pragma unroll
        for (int j = 0; j < QS_UNROLL; ++j) {
            mn = fminf(mn, q[j]);
            sm += (double)q[j];
            if (check && q[j] < lastMin - tol) ++fl;
        }
    }
    for (; e < nE; e += st) {
        const float q = element_quality(el, kind, pos, e);
        mn = fminf(mn, q);
        sm += (double)q;
        if (check && q < lastMin - tol) ++fl;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(FULL, mn, o));
        sm += __shfl_xor_sync(FULL, sm, o);
        fl += __shfl_xor_sync(FULL, fl, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { smin[w] = mn; ssum[w] = sm; sfail[w] = fl; }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = smin[0]; double s = ssum[0]; int f = sfail[0];
        for (int i = 1; i < QS_THREADS / 32; ++i) { a = fminf(a, smin[i]); s += ssum[i]; f += sfail[i]; }
        pmin[blockIdx.x] = a; psum[blockIdx.x] = s; pfail[blockIdx.x] = f;
        __threadfence();
        last = atomicAdd(done, 1u) == QS_BLOCKS - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block folds the partials: thread t takes t, t + QS_THREADS, ... in order, then a
    // fixed tree (the same order every run)
    __threadfence();
    {
        float a = FLT_MAX; double s = 0.0; int f = 0;
        for (int i = threadIdx.x; i < QS_BLOCKS; i += QS_THREADS) {
            a = fminf(a, ((volatile float*)pmin)[i]); s += ((volatile double*)psum)[i]; f += ((volatile int*)pfail)[i];
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            a = fminf(a, __shfl_xor_sync(FULL, a, o));
            s += __shfl_xor_sync(FULL, s, o);
            f += __shfl_xor_sync(FULL, f, o);
        }
        if (lane == 0) { smin[w] = a; ssum[w] = s; sfail[w] = f; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = smin[0]; double s = ssum[0]; int f = sfail[0];
        for (int i = 1; i < QS_THREADS / 32; ++i) { a = fminf(a, smin[i]); s += ssum[i]; f += sfail[i]; }
        const int slot = init ? 0 : it + 1;
        stats[slot].min_q = a;
        stats[slot].sum_q = s;
        stats[slot].fail_count = f;
        if (!init) *iter = it + 1;
        *done = 0u;
    }
}

__global__ void k_element_qualities(const int* __restrict__ el, int kind, long nE, const float4* __restrict__ pos, float* out) {
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < nE; e += (long)gridDim.x * blockDim.x)
        out[e] = element_quality(el, kind, pos, e);
}

__global__ void k_quality_histogram(const int* __restrict__ el, int kind, long nE, const float4* __restrict__ pos,
                                    int* counts, int n_cols) {
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < nE; e += (long)gridDim.x * blockDim.x) {
        float q = fminf(0.9999f, element_quality(el, kind, pos, e));
        int idx = q > 0.f ? (int)(q * n_cols) : 0;  // a negative quality lands in bin 0
        atomicAdd(&counts[idx], 1);
    }
}

}  // namespace

int dmo_tet_max_ring() { return TET_MAX_RING; }
int dmo_hex_max_ring() { return HEX_MAX_RING; }

void launch_dmo_hex(const Mesh& m, const DmoLaunch& L, cudaStream_t s) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    const int maxk = m.maxTets;
    const size_t smem = (size_t)maxk * HEX_CO * sizeof(float);
    k_dmo_hex<<<n, HEX_THREADS, smem, s>>>(m.pos.p, m.hf_rowptr.p, m.hh.p, L.v0, L.grid_scale, L.depth, maxk);
    VSDMO_CHECK_LAUNCH();
}

// coefficients of every warp's ring, then every warp's survivor list
size_t tet_smem_bytes(int maxk) { return (size_t)TET_WARPS * maxk * 2 * sizeof(float4) + (size_t)TET_WARPS * TET_LIST * sizeof(int); }

// Raises the dynamic shared-memory limit of the grid-search kernels (called once per
// optimiser, outside any stream capture, on the current device).
void prepare_dmo_kernels() {
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_tet, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tet_smem_bytes(TET_MAX_RING)));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_tri2d, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    TRI_WARPS * TRI_MAX_RING * 2 * (int)sizeof(float4)));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_tet_learned, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    TET_WARPS * TET_MAX_RING * 2 * (int)sizeof(float4)));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_tet_list, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)tet_smem_bytes(TET_MAX_RING)));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_hex, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    HEX_MAX_RING * HEX_CO * (int)sizeof(float)));
}
int dmo_tri2d_max_ring() { return TRI_MAX_RING; }
int quality_stats_blocks() { return QS_BLOCKS; }

void launch_dmo_tet(const Mesh& m, const DmoLaunch& L, cudaStream_t s, uint8_t* dirty,
                    unsigned long long* skipped) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    const int maxk = m.maxTets;
    const size_t smem = tet_smem_bytes(maxk);
    k_dmo_tet<<<(n + TET_WARPS - 1) / TET_WARPS, TET_WARPS * 32, smem, s>>>(
        m.pos.p, m.hf_rowptr.p, m.hf.p, L.v0, L.v1, L.grid_scale, L.depth, maxk, dirty, skipped);
    VSDMO_CHECK_LAUNCH();
}

// Active set with a free boundary: the boundary passes move vertices whose rings hold interior
// vertices; flagging the rings of all boundary vertices [v0, v1) keeps "skipping changes no
// result" without tracking which boundary vertex moved. One warp per vertex.
__global__ void k_mark_rings(const int* __restrict__ rowptr, const int4* __restrict__ hf, int v0, int v1,
                             uint8_t* __restrict__ dirty) {
    const int v = v0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (v >= v1) return;
    const int b = rowptr[v];
    tet_mark_ring(hf, b, rowptr[v + 1] - b, threadIdx.x & 31, dirty);
}

void launch_mark_rings(const Mesh& m, int v0, int v1, uint8_t* dirty, cudaStream_t s) {
    if (v1 <= v0 || !dirty) return;
    const long threads = 32L * (v1 - v0);
    k_mark_rings<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(m.hf_rowptr.p, m.hf.p, v0, v1, dirty);
    VSDMO_CHECK_LAUNCH();
}

void launch_tet_neighbours(const Mesh& m, int v0, int v1, int* nb, int* nbn, cudaStream_t s) {
    if (v1 <= v0) return;
    k_tet_neighbours<<<grid_for(v1 - v0, 128), 128, 0, s>>>(m.hf_rowptr.p, m.hf.p, v0, v1, nb, nbn);
    VSDMO_CHECK_LAUNCH();
}

void launch_tet_features(const Mesh& m, int v0, int v1, const int* nb, const int* nbn, int nb_base, float* feats,
                         uint8_t* packed, float* scale, float4* old, cudaStream_t s) {
    if (v1 <= v0) return;
    k_tet_features<<<grid_for(v1 - v0, 128), 128, 0, s>>>(m.pos.p, v0, v1, nb, nbn, nb_base, feats, packed, scale, old);
    VSDMO_CHECK_LAUNCH();
}

void launch_tet_targets(const Mesh& m, int v0, int v1, const float* scale, const float4* old, float* targets,
                        cudaStream_t s) {
    if (v1 <= v0) return;
    k_tet_targets<<<grid_for(v1 - v0, 256), 256, 0, s>>>(m.pos.p, v0, v1, scale, old, targets);
    VSDMO_CHECK_LAUNCH();
}

void launch_dmo_tet_learned(const Mesh& m, const DmoLaunch& L, const float* Y, int ldy, int rn, int rdepth,
                            float rscale, unsigned long long* counters, uint8_t* dirty, int* fb_list, int* fb_count,
                            cudaStream_t s) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    const int maxk = m.maxTets;
    const size_t smem = (size_t)TET_WARPS * maxk * 2 * sizeof(float4);
    k_dmo_tet_learned<<<(n + TET_WARPS - 1) / TET_WARPS, TET_WARPS * 32, smem, s>>>(
        m.pos.p, m.hf_rowptr.p, m.hf.p, L.v0, L.v1, L.grid_scale, maxk, Y, ldy, rn, rdepth, rscale, counters, dirty,
        fb_list, fb_count);
    VSDMO_CHECK_LAUNCH();
    // fallback: the plain search over the queued vertices, a fixed grid striding over the list
    const int blocks = std::min((n + TET_WARPS - 1) / TET_WARPS, 148 * 4);
    k_dmo_tet_list<<<blocks, TET_WARPS * 32, tet_smem_bytes(maxk), s>>>(m.pos.p, m.hf_rowptr.p, m.hf.p, fb_list, fb_count,
                                                                        L.grid_scale, L.depth, maxk, dirty, counters + 2);
    VSDMO_CHECK_LAUNCH();
}

void launch_dmo_tri2d(const Mesh& m, const DmoLaunch& L, cudaStream_t s) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    const int maxk = m.maxHE;
    const size_t smem = (size_t)TRI_WARPS * maxk * 2 * sizeof(float4);
    k_dmo_tri2d<<<(n + TRI_WARPS - 1) / TRI_WARPS, TRI_WARPS * 32, smem, s>>>(
        m.pos.p, m.he_rowptr.p, m.he.p, L.v0, L.v1, L.grid_scale, L.depth, maxk);
    VSDMO_CHECK_LAUNCH();
}

void launch_quality_stats(const Mesh& m, int kind, IterStats* d_stats, int* d_iter, float* d_partial_min,
                          double* d_partial_sum, int* d_partial_fail, unsigned* d_done, int check_monotone,
                          cudaStream_t s) {
    // check_monotone < 0 marks the initial evaluation (slot 0, no check, no increment)
    const int init = check_monotone < 0 ? 1 : 0;
    k_quality_stats<<<QS_BLOCKS, QS_THREADS, 0, s>>>(m.elems.p, kind, m.nE, m.pos.p, d_stats, d_iter, d_partial_min,
                                                     d_partial_sum, d_partial_fail, d_done, init ? 0 : check_monotone, init);
    VSDMO_CHECK_LAUNCH();
}

void launch_element_qualities(const Mesh& m, int kind, float* d_out, cudaStream_t s) {
    k_element_qualities<<<grid_for(m.nE, 256), 256, 0, s>>>(m.elems.p, kind, m.nE, m.pos.p, d_out);
    VSDMO_CHECK_LAUNCH();
}

void launch_quality_histogram(const Mesh& m, int kind, int* d_counts, int n_cols, cudaStream_t s) {
    k_quality_histogram<<<grid_for(m.nE, 256), 256, 0, s>>>(m.elems.p, kind, m.nE, m.pos.p, d_counts, n_cols);
    VSDMO_CHECK_LAUNCH();
}

}  // namespace vsdmo
