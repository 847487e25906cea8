// batch.cu -- many independent 2D meshes optimised together (batched DMO).
//
// A batch concatenates up to thousands of flat triangle and quad meshes of uneven size into
// one vertex / halfedge / element space and runs one DMO iteration of all of them as a single
// persistent launch:
//
//   * work items are (mesh, colour class, vertex chunk) in colour-major order over all meshes,
//     handed out by one global atomic counter; an item of colour c of mesh m waits (bounded)
//     until every vertex of colour c-1 of the same mesh is done (per-(mesh, colour) counters).
//     Items are taken only by running warps and only wait on items taken before them, so the
//     launch cannot deadlock however many CTAs are resident;
//   * every mesh carries its own search configuration -- candidates per axis (4 or 8),
//     refinement levels (1..4), lanes per vertex (8, 16 or 32: a warp searches 4, 2 or 1
//     vertices at a time) -- chosen per size bucket by the autotuner below;
//   * positions of vertices other warps may have moved during the launch are read through L2
//     (__ldcg); moves are published with __threadfence before the completion count;
//   * a second kernel reduces each mesh's element qualities (min, sum, monotonicity count).
// One iteration = memset of the counters + the two kernels, captured once as a CUDA graph and
// replayed. The grid search is the 2D search of k_optimizeHierarchical2DFlat
// (dmo/DMOTriFlatImplCub.h:24-152) generalised to N candidates per axis (oracle/or_flat.c
// restates it); with N = 8, 3 levels it is the reference kernel.
#include "vsdmo_internal.cuh"
#include "batch.cuh"
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <memory>

namespace vsdmo {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int BCO = 9;                 // coefficient floats per ring element
constexpr int BATCH_WARPS = 8;
constexpr unsigned long long BWAIT_NS = 1000000000ull;
// limit of a colour-class wait: BWAIT_NS unless the test-only vsdmo_debug_set_wait_limit_ns
// lowered it to make waits expire
__device__ unsigned long long g_batch_wait_ns = BWAIT_NS;

__device__ __forceinline__ unsigned long long bnow() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ float bexp2(int e) { return (e >= -126 && e <= 127) ? __int_as_float((e + 127) << 23) : 0.f; }
__device__ __forceinline__ float bscale(float x, float p, int e) { return p != 0.f ? x * p : ldexpf(x, e); }

template <bool COHERENT>
__device__ __forceinline__ float4 ldpos(const float4* p) {
    if (COHERENT) return __ldcg(p);
    return *p;
}

// triangle (p, a, b): A = K0 x + K1 y + K2, L = K5 + K3 x + K4 y + 2 |p|^2
__device__ __forceinline__ void btri_co(float ax, float ay, float bx, float by, float* K) {
    const float ux = bx - ax, uy = by - ay;
    K[0] = -uy; K[1] = ux;
    K[2] = ax * uy - ay * ux;
    K[3] = -2.0f * (ax + bx); K[4] = -2.0f * (ay + by);
    K[5] = ((ax * ax + ay * ay) + (bx * bx + by * by)) + (ux * ux + uy * uy);
}

// quad (p, a, b, c): corner cross products c1 = K0 x + K1 y + K2, c2 = K3 x + K4 y + K5,
// edge sum l = K8 + K6 x + K7 y + 2 |p|^2
__device__ __forceinline__ void bquad_co(float ax, float ay, float bx, float by, float cx, float cy, float* K) {
    const float e1x = bx - ax, e1y = by - ay;
    const float fx = bx - cx, fy = by - cy;
    const float gx = cx - bx, gy = cy - by;
    K[0] = -e1y; K[1] = e1x; K[2] = e1y * ax - e1x * ay;
    K[3] = fy; K[4] = -fx; K[5] = cy * fx - cx * fy;
    K[6] = -2.0f * (ax + cx); K[7] = -2.0f * (ay + cy);
    K[8] = (((ax * ax + ay * ay) + (e1x * e1x + e1y * e1y)) + (gx * gx + gy * gy)) + (cx * cx + cy * cy);
}

template <int FK>
__device__ __forceinline__ float bkey(const float* co, int k, float x, float y) {
    const float tx = (2.0f * x) * x, ty = (2.0f * y) * y;
    float N = 0.f, D = 1.f;
    if (FK == 3) {
        float amin = 0.f;
        for (int t = 0; t < k; ++t) {
            const float* c = co + BCO * t;
            const float A = fmaf(c[1], y, fmaf(c[0], x, c[2]));
            const float L = (c[5] + fmaf(c[3], x, tx)) + fmaf(c[4], y, ty);
            if (t == 0) { N = A; D = L; amin = A; continue; }
            if (A * D < N * L) { N = A; D = L; }
            amin = fminf(amin, A);
        }
        return amin < 0.f ? amin : N / D;
    } else {
        bool neg = false;
        for (int t = 0; t < k; ++t) {
            const float* c = co + BCO * t;
            const float c1 = fmaf(c[1], y, fmaf(c[0], x, c[2]));
            const float c2 = fmaf(c[4], y, fmaf(c[3], x, c[5]));
            const float l = (c[8] + fmaf(c[6], x, tx)) + fmaf(c[7], y, ty);
            neg |= (c1 < 0.f || c2 < 0.f);
            const float num = c1 + c2;
            if (t == 0) { N = num; D = l; continue; }
            if (num * D < N * l) { N = num; D = l; }
        }
        return neg ? -1.f : N / D;
    }
}

__device__ __forceinline__ float boffset(int i, int n) { return (float)(n - 1 - 2 * i) / (float)(n - 1); }

// One vertex searched by a group of L lanes (gl = lane in group, gbase = first lane of the
// group in the warp). co: the group's shared-memory coefficient buffer (maxk x BCO floats).
template <int FK, bool COHERENT>
__device__ void flat_vertex(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he,
                            int v, float gs, int nq, int depth, float* co, int maxk, int gl, int L, unsigned gmask) {
    const int b = rowptr[v], k = rowptr[v + 1] - b;
    if (k <= 0 || k > maxk) return;
    const float4 c0 = ldpos<COHERENT>(pos + v);
    float mdx = 0.f, mdy = 0.f;
    for (int t = gl; t < k; t += L) {
        const int4 h = he[b + t];
        const float4 p = ldpos<COHERENT>(pos + h.x);
        mdx = fmaxf(mdx, fabsf(p.x - c0.x)); mdy = fmaxf(mdy, fabsf(p.y - c0.y));
        if (FK == 4) {
            const float4 p2 = ldpos<COHERENT>(pos + he[h.w].x);
            mdx = fmaxf(mdx, fabsf(p2.x - c0.x)); mdy = fmaxf(mdy, fabsf(p2.y - c0.y));
        }
    }
    for (int o = L >> 1; o; o >>= 1) {
        mdx = fmaxf(mdx, __shfl_xor_sync(gmask, mdx, o, L));
        mdy = fmaxf(mdy, __shfl_xor_sync(gmask, mdy, o, L));
    }
    const float mm = fmaxf(mdx, mdy);
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return;
    int ex;
    (void)frexpf(mm, &ex);
    const float p2 = bexp2(-ex);
    for (int t = gl; t < k; t += L) {
        const int4 h = he[b + t];
        const float4 pa = ldpos<COHERENT>(pos + h.x);
        const float4 pn = ldpos<COHERENT>(pos + he[b + (t + 1 == k ? 0 : t + 1)].x);
        const float ax = bscale(pa.x - c0.x, p2, -ex), ay = bscale(pa.y - c0.y, p2, -ex);
        const float nx = bscale(pn.x - c0.x, p2, -ex), ny = bscale(pn.y - c0.y, p2, -ex);
        if (FK == 3) {
            btri_co(ax, ay, nx, ny, co + BCO * t);
        } else {
            const float4 pb = ldpos<COHERENT>(pos + he[h.w].x);
            const float bx = bscale(pb.x - c0.x, p2, -ex), by = bscale(pb.y - c0.y, p2, -ex);
            bquad_co(ax, ay, bx, by, nx, ny, co + BCO * t);
        }
    }
    __syncwarp(gmask);
    const float sx = bscale(mdx, p2, -ex), sy = bscale(mdy, p2, -ex);
    const int nvt = nq * nq / 2;
    float dx = 0.f, dy = 0.f;
    const float qOld = bkey<FK>(co, k, 0.f, 0.f);
    float qLast = qOld, lastMax = -FLT_MAX;
    float ds = gs;
    for (int level = 0; level < depth; ++level) {
        const float Sx = ds * sx, Sy = ds * sy;
        float bv = -FLT_MAX, bx = 0.f, by = 0.f;
        int bt = 1 << 30;
        for (int vt = gl; vt < nvt; vt += L) {
            const int i1 = vt / nq, j1 = vt % nq, i2 = i1 + nq / 2;
            const float x1 = fmaf(boffset(i1, nq), Sx, dx), x2 = fmaf(boffset(i2, nq), Sx, dx);
            const float y = fmaf(boffset(j1, nq), Sy, dy);
            const float q1 = bkey<FK>(co, k, x1, y), q2 = bkey<FK>(co, k, x2, y);
            float val = q1;
            if (q2 > q1) val = q2;
            if (bt == (1 << 30) || val > bv) { bv = val; bt = vt; bx = q1 > q2 ? x1 : x2; by = y; }
        }
        // group arg-max: larger value, lower virtual thread on ties
        for (int o = L >> 1; o; o >>= 1) {
            const float ov = __shfl_xor_sync(gmask, bv, o, L);
            const int ot = __shfl_xor_sync(gmask, bt, o, L);
            const float ox = __shfl_xor_sync(gmask, bx, o, L), oy = __shfl_xor_sync(gmask, by, o, L);
            if (ov > bv || (ov == bv && ot < bt)) { bv = ov; bt = ot; bx = ox; by = oy; }
        }
        if (qLast < bv) { dx = bx; dy = by; qLast = bv; }
        lastMax = bv;
        ds = ds * (2.0f / (float)(nq - 1));
    }
    if (gl == 0 && qOld < lastMax) {
        const float pu = bexp2(ex);
        pos[v] = make_float4(c0.x + bscale(dx, pu, ex), c0.y + bscale(dy, pu, ex), c0.z, c0.w);
    }
    __syncwarp(gmask);
}

// ---- single flat mesh: one colour class, one group of L lanes per vertex ------------------------
template <int FK>
__global__ void __launch_bounds__(BATCH_WARPS * 32)
k_dmo_flat(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he, int v0, int v1,
           float gs, int nq, int depth, int L, int maxk) {
    extern __shared__ float fsm[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int groups = 32 / L, g = lane / L, gl = lane % L;
    const unsigned gmask = L == 32 ? FULL : (((1u << L) - 1u) << (g * L));
    float* co = fsm + ((size_t)w * groups + g) * maxk * BCO;
    const int v = v0 + (blockIdx.x * BATCH_WARPS + w) * groups + g;
    if (v >= v1) return;
    flat_vertex<FK, false>(pos, rowptr, he, v, gs, nq, depth, co, maxk, gl, L, gmask);
}

// ---- the persistent batched iteration -----------------------------------------------------------
__global__ void __launch_bounds__(BATCH_WARPS * 32)
k_batch_iter(float4* __restrict__ pos, const int* __restrict__ rowptr, const int4* __restrict__ he,
             const BatchItem* __restrict__ items, int n_items, const BatchMeshDev* __restrict__ meshes,
             const int* __restrict__ csize, int* __restrict__ done, int* __restrict__ head, int maxk, float gs,
             int* __restrict__ err) {
    extern __shared__ float bsm[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float* wco = bsm + (size_t)w * 4 * maxk * BCO;   // up to 4 groups per warp
    while (true) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(head, 1);
        idx = __shfl_sync(FULL, idx, 0);
        if (idx >= n_items) break;
        const BatchItem it = items[idx];
        const BatchMeshDev mh = meshes[it.mesh];
        if (it.color > 0) {
            // wait (bounded) for the previous colour class of this mesh; once any wait has
            // expired nobody waits any more: the remaining items are counted and skipped
            int ok = 1;
            if (lane == 0) {
                const volatile int* d = done + mh.col_base + it.color - 1;
                const volatile int* ve = err;
                const int need = csize[mh.col_base + it.color - 1];
                if (*d < need) {
                    const unsigned long long t0 = bnow();
                    const unsigned long long lim = *(volatile unsigned long long*)&g_batch_wait_ns;
                    while (*d < need) {
                        if (*ve) { ok = 0; break; }
                        __nanosleep(128);
                        if (bnow() - t0 >= lim) { ok = 0; atomicExch(err, 1); break; }
                    }
                }
                __threadfence();
            }
            ok = __shfl_sync(FULL, ok, 0);
            if (!ok) {
                if (lane == 0) atomicAdd(done + mh.col_base + it.color, it.v1 - it.v0);
                continue;
            }
        }
        const int L = mh.lanes, groups = 32 / L, g = lane / L, gl = lane % L;
        const unsigned gmask = L == 32 ? FULL : (((1u << L) - 1u) << (g * L));
        float* co = wco + (size_t)g * maxk * BCO;
        for (int base = it.v0; base < it.v1; base += groups) {
            const int v = base + g;
            if (v < it.v1) {
                if (mh.fk == 3) flat_vertex<3, true>(pos, rowptr, he, v, gs, mh.nq, mh.depth, co, maxk, gl, L, gmask);
                else flat_vertex<4, true>(pos, rowptr, he, v, gs, mh.nq, mh.depth, co, maxk, gl, L, gmask);
            }
        }
        // publish: every writer fences its moves before lane 0 counts the chunk as done
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicAdd(done + mh.col_base + it.color, it.v1 - it.v0);
    }
}

// per-mesh element quality statistics: block m reduces mesh m
__device__ __forceinline__ float bq_tri(float4 p0, float4 p1, float4 p2) {
    const float e0x = p1.x - p0.x, e0y = p1.y - p0.y, e1x = p2.x - p1.x, e1y = p2.y - p1.y;
    const float e2x = p0.x - p2.x, e2y = p0.y - p2.y;
    const float l = ((e0x * e0x + e0y * e0y) + (e1x * e1x + e1y * e1y)) + (e2x * e2x + e2y * e2y);
    const float area = e0x * e1y - e0y * e1x;
    if (area < 0.f) return area;
    return ((2.f * sqrtf(3.f)) * area) / l;
}

__device__ __forceinline__ float bq_quad(float4 p0, float4 p1, float4 p2, float4 p3) {
    const float e0x = p1.x - p0.x, e0y = p1.y - p0.y, e1x = p2.x - p1.x, e1y = p2.y - p1.y;
    const float e2x = p3.x - p2.x, e2y = p3.y - p2.y, e3x = p0.x - p3.x, e3y = p0.y - p3.y;
    const float l = (((e0x * e0x + e0y * e0y) + (e1x * e1x + e1y * e1y)) + (e2x * e2x + e2y * e2y)) + (e3x * e3x + e3y * e3y);
    const float c1 = e1x * (-e0y) - e1y * (-e0x);
    const float c2 = e3x * (-e2y) - e3y * (-e2x);
    if (c1 < 0.f || c2 < 0.f) return -1.f;
    return (2.f * (c1 + c2)) / l;
}

__global__ void __launch_bounds__(256)
k_batch_quality(const float4* __restrict__ pos, const int* __restrict__ el, const BatchMeshDev* __restrict__ meshes,
                BatchStats* __restrict__ stats, int n_meshes, int* __restrict__ iter, int init) {
    __shared__ float smin[8];
    __shared__ double ssum[8];
    __shared__ int sfail[8];
    const int m = blockIdx.x;
    const BatchMeshDev mh = meshes[m];
    const int it = *iter;
    const float last = init ? -FLT_MAX : stats[(size_t)it * n_meshes + m].min_q;
    const float tol = 1e-6f * fmaxf(fabsf(last), 1e-30f);
    float mn = FLT_MAX;
    double sm = 0.0;
    int fl = 0;
    for (int e = threadIdx.x; e < mh.n_elems; e += 256) {
        const int* t = el + mh.el_off + (long)mh.fk * e;
        const float q = mh.fk == 3 ? bq_tri(pos[t[0]], pos[t[1]], pos[t[2]]) : bq_quad(pos[t[0]], pos[t[1]], pos[t[2]], pos[t[3]]);
        mn = fminf(mn, q);
        sm += (double)q;
        if (!init && q < last - tol) ++fl;
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
        float a = smin[0];
        double s = ssum[0];
        int f = sfail[0];
        for (int i = 1; i < 8; ++i) { a = fminf(a, smin[i]); s += ssum[i]; f += sfail[i]; }
        const int slot = init ? 0 : it + 1;
        BatchStats& o = stats[(size_t)slot * n_meshes + m];
        o.min_q = a; o.sum_q = s; o.fail_count = f;
    }
}

__global__ void k_batch_iter_advance(int* iter) { *iter += 1; }

// positions in the input numbering <-> batch numbering
__global__ void k_batch_pack(const float4* __restrict__ pos, const int* __restrict__ map, long n, float* __restrict__ out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float4 p = pos[map[i]];
        out[3 * i] = p.x; out[3 * i + 1] = p.y; out[3 * i + 2] = p.z;
    }
}

__global__ void k_batch_unpack(float4* __restrict__ pos, const int* __restrict__ map, long n, const float* __restrict__ in) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        float4& p = pos[map[i]];
        p.x = in[3 * i]; p.y = in[3 * i + 1]; p.z = in[3 * i + 2];
    }
}

// concatenation: copy one mesh's arrays into the batch with offsets applied
__global__ void k_batch_concat_he(const int4* he, int n, int v_off, int he_off, int4* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 h = he[i];
        out[i] = make_int4(h.x + v_off, h.y >= 0 ? h.y + he_off : -1, h.z, h.w + he_off);
    }
}

__global__ void k_batch_concat_int(const int* in, int n, int off, int* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[i] + off;
}

}  // namespace

// ---- host ---------------------------------------------------------------------------------------------
size_t flat_smem(int maxk, int groups) { return (size_t)BATCH_WARPS * groups * maxk * BCO * sizeof(float); }

int flat_max_ring() { return 64; }

void prepare_flat_kernels() {
    static bool done = false;
    if (done) return;
    const int mx = (int)flat_smem(flat_max_ring(), 4);
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_flat<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    VSDMO_CUDA(cudaFuncSetAttribute(k_dmo_flat<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    VSDMO_CUDA(cudaFuncSetAttribute(k_batch_iter, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    done = true;
}

void launch_dmo_flat(const Mesh& m, const DmoLaunch& L, int nq, int lanes, cudaStream_t s) {
    const int n = L.v1 - L.v0;
    if (n <= 0) return;
    if (m.maxHE > flat_max_ring()) throw Error(VSDMO_E_VALENCE, "a vertex has more halfedges than the flat kernel's ring budget");
    prepare_flat_kernels();
    const int groups = 32 / lanes;
    const int maxk = std::max(m.maxHE, 1);
    const int per_block = BATCH_WARPS * groups;
    const int blocks = (n + per_block - 1) / per_block;
    if (m.fk == 4)
        k_dmo_flat<4><<<blocks, BATCH_WARPS * 32, flat_smem(maxk, groups), s>>>(m.pos.p, m.he_rowptr.p, m.he.p, L.v0, L.v1,
                                                                                L.grid_scale, nq, L.depth, lanes, maxk);
    else
        k_dmo_flat<3><<<blocks, BATCH_WARPS * 32, flat_smem(maxk, groups), s>>>(m.pos.p, m.he_rowptr.p, m.he.p, L.v0, L.v1,
                                                                                L.grid_scale, nq, L.depth, lanes, maxk);
    VSDMO_CHECK_LAUNCH();
}

Batch::~Batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
}

void Batch::build(const std::vector<MeshInput>& inputs, uint32_t seed) {
    const int M = (int)inputs.size();
    hm.assign(M, BatchMeshHost{});
    long vtot = 0, hetot = 0, eltot = 0;
    int coltot = 0;
    maxk = 1;
    for (const MeshInput& in : inputs) vtot += in.nV;
    if (vtot > (long)INT32_MAX / 2) throw Error(VSDMO_E_ARG, "batch too large for 32-bit indices");
    nV = vtot;
    pos.alloc(vtot, stream);
    old_to_batch.alloc(vtot, stream);
    rowptr.alloc(vtot + 1, stream);
    // per-mesh builds first (connectivity, colouring); their halfedges / elements are kept
    // until the concatenated arrays can be sized
    std::vector<std::unique_ptr<Mesh>> built(M);
    vtot = 0;
    for (int i = 0; i < M; ++i) {
        const MeshInput& in = inputs[i];
        std::unique_ptr<Mesh> mp(new Mesh);
        Mesh& m = *mp;
        m.type = in.elem_type;
        m.k = in.elem_type == VSDMO_TRI ? 3 : 4;
        m.nV = in.nV;
        m.nE = in.nE;
        m.seed = seed;
        m.stream = stream;
        build_mesh(m, in.d_xyz, in.d_elems);
        if (!m.isFlat) throw Error(VSDMO_E_UNSUPPORTED, "mesh " + std::to_string(i) + " of the batch is not flat (z = 0)");
        if (m.nSurf != m.nV) throw Error(VSDMO_E_ARG, "mesh " + std::to_string(i) + " has vertices outside its elements");
        BatchMeshHost& h = hm[i];
        h.fk = m.fk;
        h.nV = m.nV;
        h.nE = m.nE;
        h.v_off = (int)vtot;
        h.he_off = (int)hetot;
        h.el_off = eltot;
        h.col_base = coltot;
        h.n_colors = m.nColFree;
        h.col = m.col_free;
        vtot += m.nV;
        hetot += m.nHE;
        eltot += (long)m.fk * m.nE;
        coltot += m.nColFree;
        maxk = std::max(maxk, m.maxHE);
        if (hetot > (long)INT32_MAX) throw Error(VSDMO_E_ARG, "batch too large for 32-bit indices");
        // positions, vertex map and halfedge rows go to the batch now
        VSDMO_CUDA(cudaMemcpyAsync(pos.p + h.v_off, m.pos.p, sizeof(float4) * m.nV, cudaMemcpyDeviceToDevice, stream));
        k_batch_concat_int<<<grid_for(m.nV, 256), 256, 0, stream>>>(m.new_of_old.p, m.nV, h.v_off, old_to_batch.p + h.v_off);
        VSDMO_CHECK_LAUNCH();
        k_batch_concat_int<<<grid_for(m.nV + 1, 256), 256, 0, stream>>>(m.he_rowptr.p, m.nV + 1, h.he_off, rowptr.p + h.v_off);
        VSDMO_CHECK_LAUNCH();
        // keep only what the concatenation below still needs
        m.tris.release(); m.hf_rowptr.release(); m.hf.release(); m.hh.release();
        m.isB1.release(); m.isFeat.release(); m.isB2.release(); m.fn.release(); m.vn.release();
        built[i] = std::move(mp);
    }
    if (maxk > flat_max_ring()) throw Error(VSDMO_E_VALENCE, "a vertex has more halfedges than the batched kernel's ring budget");
    he.alloc(std::max<long>(hetot, 1), stream);
    el.alloc(std::max<long>(eltot, 1), stream);
    std::vector<int> cs(std::max(coltot, 1), 0);
    for (int i = 0; i < M; ++i) {
        Mesh& m = *built[i];
        const BatchMeshHost& h = hm[i];
        k_batch_concat_he<<<grid_for(m.nHE, 256), 256, 0, stream>>>(m.he.p, m.nHE, h.v_off, h.he_off, he.p + h.he_off);
        VSDMO_CHECK_LAUNCH();
        k_batch_concat_int<<<grid_for((long)m.fk * m.nE, 256), 256, 0, stream>>>(m.elems.p, m.fk * m.nE, h.v_off, el.p + h.el_off);
        VSDMO_CHECK_LAUNCH();
        for (int c = 0; c < h.n_colors; ++c) cs[h.col_base + c] = h.col[c + 1] - h.col[c];
        built[i].reset();   // stream-ordered frees
    }
    csize.alloc(cs.size(), stream);
    done.alloc(cs.size(), stream);
    VSDMO_CUDA(cudaMemcpyAsync(csize.p, cs.data(), sizeof(int) * cs.size(), cudaMemcpyHostToDevice, stream));
    head.alloc(1, stream);
    err.alloc(1, stream);
    err.zero();
    d_iter.alloc(1, stream);
    d_iter.zero();
    cfg.assign(M, BatchConfig{8, 3, 32});
    d_meshes.alloc(std::max(M, 1), stream);
    upload_meshes();
    VSDMO_CUDA(cudaStreamSynchronize(stream));
}

int Batch::n_colors_total() const { return (int)csize.n; }

void Batch::upload_meshes() {
    std::vector<BatchMeshDev> dm(hm.size());
    for (size_t i = 0; i < hm.size(); ++i) {
        dm[i].fk = hm[i].fk;
        dm[i].nq = cfg[i].nq;
        dm[i].depth = cfg[i].depth;
        dm[i].lanes = cfg[i].lanes;
        dm[i].col_base = hm[i].col_base;
        dm[i].n_elems = hm[i].nE;
        dm[i].el_off = hm[i].el_off;
    }
    VSDMO_CUDA(cudaMemcpyAsync(d_meshes.p, dm.data(), sizeof(BatchMeshDev) * dm.size(), cudaMemcpyHostToDevice, stream));
    VSDMO_CUDA(cudaStreamSynchronize(stream));   // dm is a host temporary
    invalidate_graph();
}

void Batch::set_configs(const std::vector<BatchConfig>& c) {
    if (c.size() != hm.size()) throw Error(VSDMO_E_ARG, "one configuration per mesh expected");
    for (const BatchConfig& b : c) {
        if (b.nq != 4 && b.nq != 8) throw Error(VSDMO_E_ARG, "candidates per axis must be 4 or 8");
        if (b.depth < 1 || b.depth > 4) throw Error(VSDMO_E_ARG, "refinement levels must be in 1..4");
        if (b.lanes != 8 && b.lanes != 16 && b.lanes != 32) throw Error(VSDMO_E_ARG, "lanes per vertex must be 8, 16 or 32");
    }
    cfg = c;
    upload_meshes();
}

void Batch::invalidate_graph() {
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
    items_dirty = true;
}

// Work items of the meshes in `sel` (all when empty) in colour-major order: every mesh's colour
// c before any mesh's colour c + 1. A chunk is 8 steps of one warp (8 x the vertices a warp
// searches at once).
std::vector<BatchItem> Batch::make_items(const std::vector<int>& sel) const {
    std::vector<int> ms = sel;
    if (ms.empty())
        for (int i = 0; i < (int)hm.size(); ++i) ms.push_back(i);
    int maxc = 0;
    for (int i : ms) maxc = std::max(maxc, hm[i].n_colors);
    std::vector<BatchItem> items;
    for (int c = 0; c < maxc; ++c)
        for (int i : ms) {
            const BatchMeshHost& h = hm[i];
            if (c >= h.n_colors) continue;
            const int v0 = h.v_off + h.col[c], v1 = h.v_off + h.col[c + 1];
            const int chunk = 8 * (32 / cfg[i].lanes);
            for (int a = v0; a < v1; a += chunk) items.push_back(BatchItem{i, c, a, std::min(v1, a + chunk)});
        }
    return items;
}

void Batch::ensure_items() {
    if (!items_dirty) return;
    std::vector<BatchItem> it = make_items({});
    n_items = (int)it.size();
    d_items.alloc(std::max(n_items, 1), stream);
    VSDMO_CUDA(cudaMemcpyAsync(d_items.p, it.data(), sizeof(BatchItem) * it.size(), cudaMemcpyHostToDevice, stream));
    VSDMO_CUDA(cudaStreamSynchronize(stream));
    items_dirty = false;
}

void Batch::ensure_launch_setup() {
    if (blocks) return;
    prepare_flat_kernels();
    int dev = 0, sms = 148, per = 1;
    VSDMO_CUDA(cudaGetDevice(&dev));
    VSDMO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    VSDMO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_iter, BATCH_WARPS * 32, flat_smem(maxk, 4)));
    blocks = sms * std::max(per, 1);
}

void Batch::quality(BatchStats* out, int* d_it, int init, cudaStream_t s) const {
    const int M = (int)hm.size();
    k_batch_quality<<<M, 256, 0, s>>>(pos.p, el.p, d_meshes.p, out, M, d_it, init);
    VSDMO_CHECK_LAUNCH();
}

void Batch::launch_iteration(const BatchItem* d_it, int n, bool with_stats, cudaStream_t s) {
    VSDMO_CUDA(cudaMemsetAsync(done.p, 0, sizeof(int) * done.n, s));
    VSDMO_CUDA(cudaMemsetAsync(head.p, 0, sizeof(int), s));
    k_batch_iter<<<blocks, BATCH_WARPS * 32, flat_smem(maxk, 4), s>>>(pos.p, rowptr.p, he.p, d_it, n, d_meshes.p, csize.p,
                                                                     done.p, head.p, maxk, grid_scale, err.p);
    VSDMO_CHECK_LAUNCH();
    if (with_stats) {
        quality(stats.p, d_iter.p, 0, s);
        k_batch_iter_advance<<<1, 1, 0, s>>>(d_iter.p);
        VSDMO_CHECK_LAUNCH();
    }
}

void Batch::ensure_stats(int iters) {
    const int M = (int)hm.size();
    if ((long)(iters + 1) * M <= (long)stats.n) return;
    const long cap = std::max<long>((long)(iters + 1) * M, 2 * (long)stats.n);
    DBuf<BatchStats> ns(cap, stream);
    ns.zero();
    if (stats.p) VSDMO_CUDA(cudaMemcpyAsync(ns.p, stats.p, sizeof(BatchStats) * stats.n, cudaMemcpyDeviceToDevice, stream));
    stats = std::move(ns);
    invalidate_graph();
}

void Batch::restart() {
    iters_done = 0;
    ensure_stats(16);
    d_iter.zero();
    quality(stats.p, d_iter.p, 1, stream);
    VSDMO_CUDA(cudaStreamSynchronize(stream));
}

void Batch::iterate(int n) {
    ensure_launch_setup();
    ensure_stats(iters_done + n);
    ensure_items();
    if (!exec) {
        VSDMO_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            launch_iteration(d_items.p, n_items, true, stream);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        VSDMO_CUDA(cudaStreamEndCapture(stream, &graph));
        VSDMO_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    }
    for (int i = 0; i < n; ++i) VSDMO_CUDA(cudaGraphLaunch(exec, stream));
    iters_done += n;
}

void batch_set_wait_limit(unsigned long long ns) {
    VSDMO_CUDA(cudaDeviceSynchronize());
    VSDMO_CUDA(cudaMemcpyToSymbol(g_batch_wait_ns, &ns, sizeof(ns)));
    VSDMO_CUDA(cudaDeviceSynchronize());
}

void Batch::check_errors() {
    const int e = read_scalar(err.p, stream);
    if (e) {
        err.zero();
        throw Error(VSDMO_E_TIMEOUT, "batched iteration: a colour-class wait expired");
    }
}

std::vector<BatchStats> Batch::read_stats(int slot) const {
    const int M = (int)hm.size();
    std::vector<BatchStats> h(M);
    if (slot < 0 || (long)(slot + 1) * M > (long)stats.n) throw Error(VSDMO_E_ARG, "no statistics for that iteration");
    VSDMO_CUDA(cudaMemcpyAsync(h.data(), stats.p + (size_t)slot * M, sizeof(BatchStats) * M, cudaMemcpyDeviceToHost, stream));
    VSDMO_CUDA(cudaStreamSynchronize(stream));
    return h;
}

void Batch::get_positions(float* d_out) const {
    k_batch_pack<<<grid_for(nV, 256), 256, 0, stream>>>(pos.p, old_to_batch.p, nV, d_out);
    VSDMO_CHECK_LAUNCH();
}

void Batch::set_positions(const float* d_in) {
    k_batch_unpack<<<grid_for(nV, 256), 256, 0, stream>>>(pos.p, old_to_batch.p, nV, d_in);
    VSDMO_CHECK_LAUNCH();
}

// ---- autotuner ----------------------------------------------------------------------------------------
// Meshes are bucketed by free-vertex count (< 2,000 / < 10,000 / more). For each bucket the
// reference configuration (8 candidates per axis, 3 levels, 32 lanes) runs `probe_iters`
// iterations of the bucket's meshes from their current positions; its mean (over the bucket)
// of the meshes' mean quality and its minimum of their minimum quality are the target. Every
// other configuration (4 or 8 per axis, 2-4 levels, 8 / 16 / 32 lanes per vertex) runs up to
// 2 x probe_iters iterations from the same positions until it reaches the target (within
// 1e-4); the configuration with the least device time to the target wins. Timing: CUDA
// events around each iteration's launch. Positions and statistics are restored afterwards.
std::vector<std::string> Batch::autotune(int probe_iters) {
    if (probe_iters < 1) throw Error(VSDMO_E_ARG, "probe_iters must be >= 1");
    const int M = (int)hm.size();
    std::vector<std::string> report;
    ensure_launch_setup();
    DBuf<float4> saved(nV, stream);
    VSDMO_CUDA(cudaMemcpyAsync(saved.p, pos.p, sizeof(float4) * nV, cudaMemcpyDeviceToDevice, stream));
    DBuf<BatchStats> qs(M, stream);
    DBuf<int> qit(1, stream);
    qit.zero();
    std::map<int, std::vector<int>> buckets;
    for (int i = 0; i < M; ++i) {
        const int free_v = hm[i].col.empty() ? 0 : hm[i].col.back() - hm[i].col.front();
        buckets[free_v < 2000 ? 0 : (free_v < 10000 ? 1 : 2)].push_back(i);
    }
    std::vector<BatchConfig> cands;
    cands.push_back({8, 3, 32});
    for (int nq : {8, 4})
        for (int d : {2, 3, 4})
            for (int l : {32, 16, 8})
                if (!(nq == 8 && d == 3 && l == 32)) cands.push_back({nq, d, l});
    cudaEvent_t e0, e1;
    VSDMO_CUDA(cudaEventCreate(&e0));
    VSDMO_CUDA(cudaEventCreate(&e1));
    std::vector<BatchConfig> chosen = cfg;
    try {
        for (auto& kv : buckets) {
            const std::vector<int>& bm = kv.second;
            double tgt_mean = 0.0, tgt_min = 0.0, best_t = 1e30;
            BatchConfig best = cands[0];
            int best_iters = probe_iters;
            for (size_t ci = 0; ci < cands.size(); ++ci) {
                const BatchConfig c = cands[ci];
                for (int i : bm) cfg[i] = c;
                upload_meshes();
                const std::vector<BatchItem> it = make_items(bm);
                DBuf<BatchItem> dit(it.size(), stream);
                VSDMO_CUDA(cudaMemcpyAsync(dit.p, it.data(), sizeof(BatchItem) * it.size(), cudaMemcpyHostToDevice, stream));
                for (int i : bm)
                    VSDMO_CUDA(cudaMemcpyAsync(pos.p + hm[i].v_off, saved.p + hm[i].v_off, sizeof(float4) * hm[i].nV,
                                               cudaMemcpyDeviceToDevice, stream));
                const int max_it = ci == 0 ? probe_iters : 2 * probe_iters;
                double t = 0.0;
                bool reached = false;
                int used = 0;
                for (int r = 0; r < max_it; ++r) {
                    VSDMO_CUDA(cudaEventRecord(e0, stream));
                    launch_iteration(dit.p, (int)it.size(), false, stream);
                    VSDMO_CUDA(cudaEventRecord(e1, stream));
                    quality(qs.p, qit.p, 1, stream);
                    std::vector<BatchStats> st(M);
                    VSDMO_CUDA(cudaMemcpyAsync(st.data(), qs.p, sizeof(BatchStats) * M, cudaMemcpyDeviceToHost, stream));
                    VSDMO_CUDA(cudaStreamSynchronize(stream));
                    float ms = 0.f;
                    VSDMO_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    t += ms;
                    used = r + 1;
                    double mean_q = 0.0, min_q = 1e30;
                    for (int i : bm) { mean_q += st[i].sum_q / std::max(hm[i].nE, 1); min_q = std::min(min_q, (double)st[i].min_q); }
                    mean_q /= (double)bm.size();
                    if (ci == 0) {
                        if (r + 1 == max_it) { tgt_mean = mean_q; tgt_min = min_q; reached = true; }
                    } else if (mean_q >= tgt_mean - 1e-4 && min_q >= tgt_min - 1e-4) {
                        reached = true;
                        break;
                    }
                }
                check_errors();
                if (reached && t < best_t) { best_t = t; best = c; best_iters = used; }
            }
            for (int i : bm) { cfg[i] = best; chosen[i] = best; }
            for (int i : bm)
                VSDMO_CUDA(cudaMemcpyAsync(pos.p + hm[i].v_off, saved.p + hm[i].v_off, sizeof(float4) * hm[i].nV,
                                           cudaMemcpyDeviceToDevice, stream));
            char line[256];
            snprintf(line, sizeof line, "bucket %d: %zu meshes, N=%d depth=%d lanes=%d, %d iterations %.3f ms to the target",
                     kv.first, bm.size(), best.nq, best.depth, best.lanes, best_iters, best_t);
            report.push_back(line);
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    VSDMO_CUDA(cudaMemcpyAsync(pos.p, saved.p, sizeof(float4) * nV, cudaMemcpyDeviceToDevice, stream));
    cfg = chosen;
    upload_meshes();
    VSDMO_CUDA(cudaStreamSynchronize(stream));
    return report;
}

}  // namespace vsdmo
